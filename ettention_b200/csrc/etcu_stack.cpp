// Directory image stacks with metadata.xml and XML parameter files, host side (no
// device code).
//
// Behaviour follows (paths relative to ettention/libReconstruction/src):
//   io/datasource/ImageStackDirectoryDatasource.cpp:23-45    loading, logscale -> exp
//   io/datasource/ImageStackDirectoryDatasource.cpp:121-175  writeMetaDataFile
//   io/datasource/ImageStackDirectoryDatasource.cpp:177-245  readMetaDataFile: projection
//       and projectionstack nodes, numbering by tilt angle, base parallel geometry
//   setup/parametersource/XMLParameterSource.cpp             value attributes by path
//
// The reference reads both files with Boost.PropertyTree's XML reader, which takes
// several top-level elements in one file.  The reader here covers what those files
// use: elements, attributes (single or double quotes, the five named entities and
// character references), comments, processing instructions, a DOCTYPE and CDATA;
// text content is ignored.
#include <algorithm>
#include <atomic>
#include <cctype>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <sstream>
#include <thread>

#include "io_util.hpp"

using etcu_io::fail;

namespace {

struct XmlNode {
    std::string name;
    std::vector<std::pair<std::string, std::string>> attrs;
    std::vector<XmlNode> children;

    const XmlNode* child(const std::string& n) const {
        for (const XmlNode& c : children)
            if (c.name == n) return &c;
        return nullptr;
    }
    const std::string* attr(const std::string& n) const {
        for (const auto& a : attrs)
            if (a.first == n) return &a.second;
        return nullptr;
    }
};

class XmlReader {
public:
    explicit XmlReader(const std::string& text) : s_(text) {}

    // The document's top-level elements become the children of `root`.
    bool read(XmlNode& root) {
        for (;;) {
            if (!skip_markup()) return false;
            if (i_ >= s_.size()) return true;
            if (s_[i_] != '<') return error("text outside an element");
            XmlNode node;
            if (!element(node, 0)) return false;
            root.children.push_back(std::move(node));
        }
    }
    const std::string& message() const { return err_; }

private:
    const std::string& s_;
    size_t i_ = 0;
    std::string err_;

    bool error(const char* what) {
        size_t line = 1;
        for (size_t k = 0; k < i_ && k < s_.size(); ++k) line += s_[k] == '\n';
        err_ = std::string(what) + " (line " + std::to_string(line) + ")";
        return false;
    }
    bool starts(const char* t) const { return s_.compare(i_, std::strlen(t), t) == 0; }
    void ws() {
        while (i_ < s_.size() && (s_[i_] == ' ' || s_[i_] == '\t' || s_[i_] == '\r' || s_[i_] == '\n')) ++i_;
    }
    bool skip_past(const char* end) {
        const size_t k = s_.find(end, i_);
        if (k == std::string::npos) return error("unterminated markup");
        i_ = k + std::strlen(end);
        return true;
    }
    // Whitespace, comments, processing instructions and DOCTYPE between elements.
    bool skip_markup() {
        for (;;) {
            ws();
            if (starts("<?")) {
                if (!skip_past("?>")) return false;
            } else if (starts("<!--")) {
                if (!skip_past("-->")) return false;
            } else if (starts("<!DOCTYPE")) {
                if (!skip_past(">")) return false;
            } else {
                return true;
            }
        }
    }
    static bool name_char(char c, bool first) {
        return std::isalpha((unsigned char)c) || c == '_' || c == ':' ||
               (!first && (std::isdigit((unsigned char)c) || c == '-' || c == '.'));
    }
    bool name(std::string& out) {
        const size_t b = i_;
        if (i_ >= s_.size() || !name_char(s_[i_], true)) return error("expected a name");
        while (i_ < s_.size() && name_char(s_[i_], false)) ++i_;
        out.assign(s_, b, i_ - b);
        return true;
    }
    static void put_utf8(std::string& out, unsigned long cp) {
        if (cp < 0x80) {
            out += char(cp);
        } else if (cp < 0x800) {
            out += char(0xC0 | (cp >> 6));
            out += char(0x80 | (cp & 0x3F));
        } else if (cp < 0x10000) {
            out += char(0xE0 | (cp >> 12));
            out += char(0x80 | ((cp >> 6) & 0x3F));
            out += char(0x80 | (cp & 0x3F));
        } else {
            out += char(0xF0 | (cp >> 18));
            out += char(0x80 | ((cp >> 12) & 0x3F));
            out += char(0x80 | ((cp >> 6) & 0x3F));
            out += char(0x80 | (cp & 0x3F));
        }
    }
    bool decode(const std::string& raw, std::string& out) {
        out.clear();
        for (size_t k = 0; k < raw.size(); ++k) {
            if (raw[k] != '&') {
                out += raw[k];
                continue;
            }
            const size_t semi = raw.find(';', k);
            if (semi == std::string::npos) return error("unterminated entity");
            const std::string ent = raw.substr(k + 1, semi - k - 1);
            if (ent == "lt") out += '<';
            else if (ent == "gt") out += '>';
            else if (ent == "amp") out += '&';
            else if (ent == "quot") out += '"';
            else if (ent == "apos") out += '\'';
            else if (ent.size() > 1 && ent[0] == '#') {
                char* end = nullptr;
                const bool hex = ent[1] == 'x' || ent[1] == 'X';
                const unsigned long cp = std::strtoul(ent.c_str() + (hex ? 2 : 1), &end, hex ? 16 : 10);
                if (!end || *end || cp == 0 || cp > 0x10FFFF) return error("invalid character reference");
                put_utf8(out, cp);
            } else {
                return error("unknown entity");
            }
            k = semi;
        }
        return true;
    }
    bool element(XmlNode& node, int depth) {
        if (depth > 256) return error("elements nested too deeply");
        ++i_;  // '<'
        if (!name(node.name)) return false;
        for (;;) {
            ws();
            if (i_ >= s_.size()) return error("unterminated start tag");
            if (starts("/>")) {
                i_ += 2;
                return true;
            }
            if (s_[i_] == '>') {
                ++i_;
                break;
            }
            std::string an, raw, val;
            if (!name(an)) return false;
            ws();
            if (i_ >= s_.size() || s_[i_] != '=') return error("expected '=' after an attribute name");
            ++i_;
            ws();
            if (i_ >= s_.size() || (s_[i_] != '"' && s_[i_] != '\'')) return error("expected a quoted value");
            const char q = s_[i_++];
            const size_t e = s_.find(q, i_);
            if (e == std::string::npos) return error("unterminated attribute value");
            raw.assign(s_, i_, e - i_);
            i_ = e + 1;
            if (!decode(raw, val)) return false;
            node.attrs.emplace_back(std::move(an), std::move(val));
        }
        for (;;) {  // content
            const size_t lt = s_.find('<', i_);
            if (lt == std::string::npos) return error("unterminated element");
            i_ = lt;
            if (starts("</")) {
                i_ += 2;
                std::string en;
                if (!name(en)) return false;
                if (en != node.name) return error("mismatched end tag");
                ws();
                if (i_ >= s_.size() || s_[i_] != '>') return error("unterminated end tag");
                ++i_;
                return true;
            }
            if (starts("<!--")) {
                if (!skip_past("-->")) return false;
            } else if (starts("<![CDATA[")) {
                if (!skip_past("]]>")) return false;
            } else if (starts("<?")) {
                if (!skip_past("?>")) return false;
            } else {
                XmlNode c;
                if (!element(c, depth + 1)) return false;
                node.children.push_back(std::move(c));
            }
        }
    }
};

etcu_status read_xml_file(const char* path, XmlNode& root) {
    std::vector<uint8_t> bytes;
    if (!etcu_io::read_file(path, bytes)) return fail(ETCU_ERR_INVALID_ARGUMENT, "%s: cannot open file", path);
    const std::string text(bytes.begin(), bytes.end());
    XmlReader r(text);
    if (!r.read(root)) return fail(ETCU_ERR_INVALID_ARGUMENT, "%s: %s", path, r.message().c_str());
    return ETCU_OK;
}

// A property-tree translation of a value: the whole string must be consumed.
template <int N>
bool parse_floats(const std::string& s, float (&out)[N]) {
    std::istringstream in(s);
    for (int k = 0; k < N; ++k)
        if (!(in >> out[k])) return false;
    in >> std::ws;
    return in.eof();
}

etcu_status value_of(const XmlNode& parent, const char* child, const char* attr, const char* file,
                     const std::string*& out) {
    const XmlNode* c = parent.child(child);
    if (!c) return fail(ETCU_ERR_INVALID_ARGUMENT, "%s: No such node (%s)", file, child);
    out = c->attr(attr);
    if (!out) return fail(ETCU_ERR_INVALID_ARGUMENT, "%s: No such node (%s.<xmlattr>.%s)", file, child, attr);
    return ETCU_OK;
}

std::string xml_escape(const std::string& s) {
    std::string o;
    for (char c : s) {
        switch (c) {
        case '&': o += "&amp;"; break;
        case '<': o += "&lt;"; break;
        case '>': o += "&gt;"; break;
        case '"': o += "&quot;"; break;
        default: o += c;
        }
    }
    return o;
}

std::string fmt_floats(const float* v, int n) {
    std::string o;
    char buf[32];
    for (int k = 0; k < n; ++k) {
        std::snprintf(buf, sizeof(buf), "%.9g", double(v[k]));
        if (k) o += ' ';
        o += buf;
    }
    return o;
}

}  // namespace

struct etcu_image_stack {
    struct Item {
        std::string file;  // relative to the directory
        int page;          // -1: a single image, else the page of a multi-page file
        float tilt;
        bool logscale;
    };
    std::string directory;
    std::vector<Item> items;  // in projection-index order
    uint32_t width = 0, height = 0;
    etcu_view base{};
};

namespace {

std::string join_path(const std::string& dir, const std::string& rel) {
    if (!rel.empty() && rel[0] == '/') return rel;
    if (dir.empty()) return rel;
    return dir.back() == '/' ? dir + rel : dir + "/" + rel;
}

// One projection decoded into `out` (height * width floats).
etcu_status load_item(const etcu_image_stack& st, const etcu_image_stack::Item& it, float* out) {
    const std::string path = join_path(st.directory, it.file);
    std::vector<uint8_t> file;
    if (!etcu_io::read_file(path.c_str(), file))
        return fail(ETCU_ERR_INVALID_ARGUMENT, "unable to load image %s", path.c_str());
    uint32_t w, h;
    std::vector<float> px;
    const etcu_status s = etcu_io::tiff_decode_page(file, path.c_str(), it.page < 0 ? 0u : uint32_t(it.page), &w, &h, px);
    if (s != ETCU_OK) return s;
    if (w != st.width || h != st.height)
        return fail(ETCU_ERR_INVALID_ARGUMENT, "image %s is %u x %u, the stack's projections are %u x %u",
                    path.c_str(), w, h, st.width, st.height);
    if (it.logscale)  // Image::convertToLinearScale
        for (float& v : px) v = std::exp(v);
    std::memcpy(out, px.data(), px.size() * sizeof(float));
    return ETCU_OK;
}

}  // namespace

extern "C" etcu_status etcu_image_stack_open(const char* directory, etcu_image_stack** out) {
    if (!directory || !out) return fail(ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    *out = nullptr;
    auto st = std::make_unique<etcu_image_stack>();
    st->directory = directory;
    const std::string meta = join_path(st->directory, "metadata.xml");
    XmlNode root;
    etcu_status s = read_xml_file(meta.c_str(), root);
    if (s != ETCU_OK) return s;
    std::vector<etcu_image_stack::Item> temp;
    for (const XmlNode& n : root.children) {
        if (n.name != "projection" && n.name != "projectionstack") continue;
        const std::string *fname, *tilt;
        if ((s = value_of(n, "image", "filename", meta.c_str(), fname)) != ETCU_OK) return s;
        if ((s = value_of(n, "tiltAngle", "value", meta.c_str(), tilt)) != ETCU_OK) return s;
        float a[1];
        if (!parse_floats(*tilt, a))
            return fail(ETCU_ERR_INVALID_ARGUMENT, "%s: conversion of data to type \"f\" failed (%s)", meta.c_str(),
                        tilt->c_str());
        const bool logscale = n.child("logscale") != nullptr;
        if (n.name == "projection") {
            temp.push_back({*fname, -1, a[0], logscale});
        } else {  // every page of a multi-page image, one tilt angle
            const std::string path = join_path(st->directory, *fname);
            std::vector<uint8_t> file;
            if (!etcu_io::read_file(path.c_str(), file))
                return fail(ETCU_ERR_INVALID_ARGUMENT, "unable to open image stack %s", path.c_str());
            uint32_t pages;
            if ((s = etcu_io::tiff_page_count(file, path.c_str(), &pages)) != ETCU_OK) return s;
            for (uint32_t p = 0; p < pages; ++p) temp.push_back({*fname, int(p), a[0], logscale});
        }
    }
    if (temp.empty()) return fail(ETCU_ERR_INVALID_ARGUMENT, "%s lists no projections", meta.c_str());
    // (index of the tilt angle in order of first appearance, repeat) -> item, in
    // lexicographic order; with unique angles this is the file's order.
    std::map<float, uint32_t> angle_index, repeats;
    std::map<std::pair<uint32_t, uint32_t>, size_t> order;
    for (size_t k = 0; k < temp.size(); ++k) {
        const float t = temp[k].tilt;
        auto f = angle_index.find(t);
        if (f == angle_index.end()) {
            f = angle_index.emplace(t, uint32_t(angle_index.size())).first;
            repeats[t] = 0;
        }
        order[{f->second, repeats[t]++}] = k;
    }
    for (const auto& o : order) st->items.push_back(temp[o.second]);
    const XmlNode* g = root.child("geometry");
    if (!g) return fail(ETCU_ERR_INVALID_ARGUMENT, "%s: No such node (geometry)", meta.c_str());
    const char* keys[4] = {"sourcePosition", "detectorPosition", "horizontalPitch", "verticalPitch"};
    float* dst[4] = {st->base.source, st->base.detector, st->base.hpitch, st->base.vpitch};
    for (int k = 0; k < 4; ++k) {
        const std::string* v;
        if ((s = value_of(*g, keys[k], "value", meta.c_str(), v)) != ETCU_OK) return s;
        float xyz[3];
        if (!parse_floats(*v, xyz))
            return fail(ETCU_ERR_INVALID_ARGUMENT, "%s: conversion of data to a vector failed (%s = \"%s\")",
                        meta.c_str(), keys[k], v->c_str());
        std::memcpy(dst[k], xyz, sizeof(xyz));
    }
    {  // detector size: the first projection's
        const auto& it = st->items.front();
        const std::string path = join_path(st->directory, it.file);
        etcu_image_info info;
        if ((s = etcu_tiff_read_info(path.c_str(), it.page < 0 ? 0u : uint32_t(it.page), &info)) != ETCU_OK) return s;
        st->width = info.width;
        st->height = info.height;
    }
    st->base.width = st->width;
    st->base.height = st->height;
    st->base.perspective = 0;
    *out = st.release();
    return ETCU_OK;
}

extern "C" void etcu_image_stack_destroy(etcu_image_stack* stack) { delete stack; }

extern "C" etcu_status etcu_image_stack_info_get(const etcu_image_stack* stack, etcu_image_stack_info* out) {
    if (!stack || !out) return fail(ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    out->count = uint32_t(stack->items.size());
    out->width = stack->width;
    out->height = stack->height;
    out->base = stack->base;
    return ETCU_OK;
}

extern "C" etcu_status etcu_image_stack_tilt_angles(const etcu_image_stack* stack, float* out, uint32_t capacity) {
    if (!stack || !out) return fail(ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    if (capacity < stack->items.size())
        return fail(ETCU_ERR_INVALID_ARGUMENT, "output holds %u of %zu tilt angles", capacity, stack->items.size());
    for (size_t k = 0; k < stack->items.size(); ++k) out[k] = stack->items[k].tilt;
    return ETCU_OK;
}

// Images are decoded on up to 16 host threads (one image per task).
extern "C" etcu_status etcu_image_stack_load(const etcu_image_stack* stack, uint32_t first, uint32_t count, float* out,
                                            size_t capacity) {
    if (!stack || (!out && count)) return fail(ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    if (uint64_t(first) + count > stack->items.size())
        return fail(ETCU_ERR_INVALID_ARGUMENT, "There is no projection for index %llu!",
                    (unsigned long long)(uint64_t(first) + count - 1));
    const size_t px = size_t(stack->width) * stack->height;
    if (capacity < px * count)
        return fail(ETCU_ERR_INVALID_ARGUMENT, "output holds %zu of %zu values", capacity, px * count);
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const unsigned nt = std::min<unsigned>({hw, 16u, std::max(1u, count)});
    std::atomic<uint32_t> next{0};
    std::vector<etcu_status> status(nt, ETCU_OK);
    std::vector<std::string> message(nt);
    std::vector<uint32_t> failed_at(nt, UINT32_MAX);
    auto work = [&](unsigned t) {
        for (uint32_t k; (k = next.fetch_add(1)) < count;) {
            const etcu_status s = load_item(*stack, stack->items[first + k], out + px * k);
            if (s != ETCU_OK) {  // the message lives in this thread's error slot
                status[t] = s;
                message[t] = etcu_last_error(nullptr);
                failed_at[t] = k;
                return;
            }
        }
    };
    if (nt == 1) {
        work(0);
    } else {
        std::vector<std::thread> pool;
        for (unsigned t = 0; t < nt; ++t) pool.emplace_back(work, t);
        for (auto& th : pool) th.join();
    }
    unsigned worst = nt;
    for (unsigned t = 0; t < nt; ++t)
        if (status[t] != ETCU_OK && (worst == nt || failed_at[t] < failed_at[worst])) worst = t;
    if (worst != nt) {
        etcu_set_context_free_error(message[worst].c_str());
        return status[worst];
    }
    return ETCU_OK;
}

extern "C" etcu_status etcu_image_stack_write_metadata(const char* path, const float* tilt_angles,
                                                     const char* const* filenames, uint32_t count,
                                                     const etcu_view* base, const uint32_t volume_resolution[3]) {
    if (!path || !base || !volume_resolution || (count && (!tilt_angles || !filenames)))
        return fail(ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    std::string o = "<?xml version=\"1.0\" encoding=\"utf-8\"?>\n<geometry>\n";
    auto vec = [&](const char* key, const float* v) {
        o += std::string("    <") + key + " value=\"" + fmt_floats(v, 3) + "\"/>\n";
    };
    vec("detectorPosition", base->detector);
    vec("sourcePosition", base->source);
    vec("horizontalPitch", base->hpitch);
    vec("verticalPitch", base->vpitch);
    o += "    <volumeDimensions value=\"" + std::to_string(volume_resolution[0]) + " " +
         std::to_string(volume_resolution[1]) + " " + std::to_string(volume_resolution[2]) + "\"/>\n</geometry>\n";
    for (uint32_t k = 0; k < count; ++k) {
        if (!filenames[k]) return fail(ETCU_ERR_INVALID_ARGUMENT, "file name %u is NULL", k);
        o += "<projection>\n    <image filename=\"" + xml_escape(filenames[k]) + "\"/>\n    <tiltAngle value=\"" +
             fmt_floats(tilt_angles + k, 1) + "\"/>\n</projection>\n";
    }
    FILE* fp = std::fopen(path, "wb");
    if (!fp) return fail(ETCU_ERR_INVALID_ARGUMENT, "Failed to open output file %s for writing!", path);
    const bool ok = std::fwrite(o.data(), 1, o.size(), fp) == o.size();
    if ((std::fclose(fp) != 0) || !ok)
        return fail(ETCU_ERR_INVALID_ARGUMENT, "Error encountered while writing to output file %s !", path);
    return ETCU_OK;
}

extern "C" etcu_status etcu_xml_config_read(const char* path, char* out, size_t capacity, size_t* needed) {
    if (!path || !needed) return fail(ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    XmlNode root;
    const etcu_status s = read_xml_file(path, root);
    if (s != ETCU_OK) return s;
    std::string text;
    std::vector<std::string> seen;
    struct Walk {
        std::string& text;
        std::vector<std::string>& seen;
        void operator()(const XmlNode& n, const std::string& prefix) {
            const std::string key = prefix.empty() ? n.name : prefix + "." + n.name;
            const std::string* v = n.attr("value");
            if (v && std::find(seen.begin(), seen.end(), key) == seen.end()) {
                seen.push_back(key);
                text += key + "\t" + *v + "\n";
            }
            children(n, key);
        }
        // Only the first element of each name is reachable by path.
        void children(const XmlNode& n, const std::string& key) {
            std::vector<std::string> names;
            for (const XmlNode& c : n.children) {
                if (std::find(names.begin(), names.end(), c.name) != names.end()) continue;
                names.push_back(c.name);
                (*this)(c, key);
            }
        }
    } walk{text, seen};
    walk.children(root, "");
    *needed = text.size() + 1;
    if (out && capacity >= text.size() + 1) std::memcpy(out, text.c_str(), text.size() + 1);
    else if (out && capacity) return fail(ETCU_ERR_INVALID_ARGUMENT, "output holds %zu of %zu bytes", capacity, text.size() + 1);
    return ETCU_OK;
}
