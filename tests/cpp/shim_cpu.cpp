// Host-only checks of include/ettention_b200.hpp: geometry, configuration keys and
// error mapping.  Prints one "key value..." line per result for tests/test_cpp_shim.py.
#include <cstdio>
#include <map>
#include <string>

#include "ettention_b200.hpp"

using namespace ettention::b200;

static void config_case(const char* name, const std::map<std::string, std::string>& cfg) {
    try {
        AlgebraicParameterSet p = AlgebraicParameterSet::fromConfig(cfg);
        std::printf("config %s ok %u %u %g %d %u\n", name, p.blockSize, p.iterations, p.lambda, (int)p.order,
                    p.subVolumeCount);
    } catch (const Exception& e) {
        std::printf("config %s error %d %s\n", name, (int)e.status(), e.what());
    }
}

int main(int argc, char** argv) {
    const ScannerGeometry g = ScannerGeometry::mrcBase(96, 80).rotated(30.f);
    const auto m = g.getProjectionMatrix();
    std::printf("matrix");
    for (float v : m) std::printf(" %.9g", v);
    std::printf("\n");
    const float lo[3] = {-48.f, -40.f, -20.f}, hi[3] = {48.f, 40.f, 20.f};
    std::printf("traversal %.9g\n", g.getTraversalLengthThroughBoundingBox(lo, hi));
    config_case("sart", {{"algorithm", "sart"}, {"algorithm.numberOfIterations", "5"}, {"algorithm.lambda", "0.3"},
                         {"optimization.projectionIteration", "identity"}});
    config_case("sirt", {{"algorithm", "sirt"}, {"algorithm.numberOfIterations", "3"}, {"algorithm.lambda", "0.5"}});
    config_case("block", {{"algorithm", "blockIterative"}, {"algorithm.blockSize", "8"},
                          {"algorithm.numberOfIterations", "2"}, {"algorithm.lambda", "0.2"},
                          {"optimization.projectionIteration", "maxangle"}, {"hardware.subVolumeCount", "3"}});
    config_case("zero_block", {{"algorithm", "blockIterative"}, {"algorithm.blockSize", "0"},
                               {"algorithm.numberOfIterations", "1"}, {"algorithm.lambda", "0.2"}});
    config_case("bad_order", {{"algorithm", "sart"}, {"optimization.projectionIteration", "zigzag"}});
    config_case("missing", {{"algorithm.lambda", "0.2"}});
    {  // files: a 4 x 3 x 2 volume written in XZY order reads back as sections y, rows z
        std::vector<float> vol(24);
        for (int i = 0; i < 24; ++i) vol[i] = (float)i;
        const char* path = argc > 1 ? argv[1] : "shim_cpu_volume.mrc";
        writeMrcVolume(path, vol.data(), {{4, 3, 2}});
        MRCStack st(path);
        const std::vector<float> back = st.loadProjections();
        bool ok = st.getNumberOfProjections() == 3 && st.getResolution()[0] == 4 && st.getResolution()[1] == 2;
        for (int y = 0; y < 3; ++y)
            for (int z = 0; z < 2; ++z)
                for (int x = 0; x < 4; ++x) ok &= back[(y * 2 + z) * 4 + x] == vol[(z * 3 + y) * 4 + x];
        std::printf("mrc %s %g %g\n", ok ? "ok" : "mismatch", st.info().dmin, st.info().dmax);
        try {
            MRCStack missing(std::string(path) + ".absent");
        } catch (const Exception& e) {
            std::printf("mrc_missing error %d\n", (int)e.status());
        }
        // a directory stack of two TIFF projections with metadata.xml, and a parameter file
        const std::string dir = std::string(path) + ".d";
        std::vector<float> img(6 * 5);
        for (int i = 0; i < 30; ++i) img[i] = 0.25f * (float)i;
        writeTiff(dir + "_p0.tif", img.data(), 6, 5);
        for (float& v : img) v = -v;
        writeTiff(dir + "_p1.tif", img.data(), 6, 5);
        const std::string base_name = dir.substr(dir.rfind('/') + 1);
        ImageStackDirectoryDatasource::writeMetaDataFile(dir.substr(0, dir.rfind('/') + 1) + "metadata.xml",
                                                         {-30.f, 45.5f}, {base_name + "_p0.tif", base_name + "_p1.tif"},
                                                         ScannerGeometry::mrcBase(6, 5), {{6, 6, 4}});
        ImageStackDirectoryDatasource ds(dir.substr(0, dir.rfind('/')));
        const std::vector<float> pr = ds.loadProjections();
        std::printf("stack %u %u %u %g %g %g %g\n", ds.getNumberOfProjections(), ds.getResolution()[0],
                    ds.getResolution()[1], ds.tiltAngles()[0], ds.tiltAngles()[1], pr[7], pr[30 + 7]);
        uint32_t w = 0, h = 0;
        const std::vector<float> t0 = readTiff(dir + "_p0.tif", 0, &w, &h);
        std::printf("tiff %u %u %g\n", w, h, t0[29]);
        const std::string xml = dir + "_run.xml";
        if (FILE* f = std::fopen(xml.c_str(), "w")) {
            std::fputs("<?xml version=\"1.0\"?>\n<algorithm value=\"sirt\"><numberOfIterations value=\"4\"/>"
                       "<lambda value=\"0.5\"/></algorithm><input><projections value=\"sub\\dir\"/></input>\n",
                       f);
            std::fclose(f);
        }
        const std::vector<float> blob = BlobParameters::createDefault().rayIntegrationSamples(4);
        std::printf("blob %.6f %.6f %.6f\n", blob[0], blob[1], blob[3]);
        XMLParameterSource src(xml);
        const auto p = AlgebraicParameterSet::fromConfig(src.values());
        const std::string proj = src.getPathParameter("input.projections");
        std::printf("xml %s %u %g %s\n", p.algorithm.c_str(), p.iterations, p.lambda,
                    proj.substr(proj.size() - 8).c_str());
    }
    try {
        Framework fw(0);
        std::printf("framework ok\n");
    } catch (const GPUException& e) {
        std::printf("framework gpu_error %d %s\n", (int)e.status(), e.what());
    } catch (const Exception& e) {
        std::printf("framework error %d %s\n", (int)e.status(), e.what());
    }
    return 0;
}
