// Forward projection, back projection and SART through include/ettention_b200.hpp on
// one GPU.  Writes raw float32 results into the directory given as argv[1] for
// tests/test_gpu_cpp_shim.py, which compares them with the oracle.
#include <cuda_runtime.h>

#include <cstdio>
#include <vector>

#include "ettention_b200.hpp"

using namespace ettention::b200;

static const uint32_t X = 96, Y = 80, Z = 40, NV = 15;

// Deterministic phantom, mirrored in the Python test.
static std::vector<float> phantom() {
    std::vector<float> v((size_t)X * Y * Z);
    for (uint32_t z = 0; z < Z; ++z)
        for (uint32_t y = 0; y < Y; ++y)
            for (uint32_t x = 0; x < X; ++x)
                v[((size_t)z * Y + y) * X + x] = 0.01f * (float)((x * 7 + y * 13 + z * 29) % 17) / 16.f;
    return v;
}

static void save(const std::string& dir, const char* name, const float* p, size_t n) {
    FILE* f = std::fopen((dir + "/" + name).c_str(), "wb");
    std::fwrite(p, sizeof(float), n, f);
    std::fclose(f);
}

static void cuda(cudaError_t e) {
    if (e != cudaSuccess) throw GPUException(ETCU_ERR_CUDA, cudaGetErrorString(e));
}

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    const std::string dir = argv[1];
    try {
        Framework fw(0);
        const std::vector<float> vol_h = phantom();
        const size_t P = (size_t)X * Y;
        float *dv = nullptr, *dl = nullptr, *dr = nullptr;
        cuda(cudaMalloc(&dv, P * 4));
        cuda(cudaMalloc(&dl, P * 4));
        cuda(cudaMalloc(&dr, P * 4));
        // forward projection of one view (two sub-volumes accumulated)
        GPUMappedVolume vol(fw, {X, Y, Z}, ETCU_VOXEL_FLOAT32, 2);
        vol.upload(vol_h.data());
        ForwardProjectionOperator fp(vol, 1);
        fp.setScannerGeometry(ScannerGeometry::mrcBase(X, Y).rotated(25.f));
        cuda(cudaMemset(dv, 0, P * 4));
        cuda(cudaMemset(dl, 0, P * 4));
        fp.SetOutput(dv, dl);
        for (uint32_t s = 0; s < vol.getSubVolumeCount(); ++s) fp.Execute(s);
        std::vector<float> pv(P), pl(P);
        cuda(cudaMemcpy(pv.data(), dv, P * 4, cudaMemcpyDeviceToHost));
        cuda(cudaMemcpy(pl.data(), dl, P * 4, cudaMemcpyDeviceToHost));
        save(dir, "fp_virtual.bin", pv.data(), P);
        save(dir, "fp_length.bin", pl.data(), P);
        // back projection of a residual image into a zero volume
        std::vector<float> res(P);
        for (size_t i = 0; i < P; ++i) res[i] = (float)((int)(i * 37 % 101) - 50) / 50.f;
        cuda(cudaMemcpy(dr, res.data(), P * 4, cudaMemcpyHostToDevice));
        GPUMappedVolume bvol(fw, {X, Y, Z});
        BackProjectionOperator bp(bvol, 0.5f, 1);
        bp.setScannerGeometry(ScannerGeometry::mrcBase(X, Y).rotated(25.f));
        bp.setInput(dr, dl, 1);
        bp.execute();
        save(dir, "bp_volume.bin", bvol.download().data(), bvol.voxelCount());
        // SART from the reference's configuration keys, 15 views over +-60 degrees
        std::vector<ScannerGeometry> views;
        std::vector<float> projs(NV * P);
        for (uint32_t i = 0; i < NV; ++i) {
            views.push_back(ScannerGeometry::mrcBase(X, Y).rotated(-60.f + 120.f * i / (NV - 1)));
            fp.setScannerGeometry(views.back());
            cuda(cudaMemset(dv, 0, P * 4));
            cuda(cudaMemset(dl, 0, P * 4));
            for (uint32_t s = 0; s < vol.getSubVolumeCount(); ++s) fp.Execute(s);
            cuda(cudaMemcpy(projs.data() + i * P, dv, P * 4, cudaMemcpyDeviceToHost));
        }
        save(dir, "projections.bin", projs.data(), projs.size());
        const AlgebraicParameterSet p = AlgebraicParameterSet::fromConfig(
            {{"algorithm", "sart"}, {"algorithm.numberOfIterations", "2"}, {"algorithm.lambda", "0.3"},
             {"optimization.projectionIteration", "identity"}});
        GPUMappedVolume rvol(fw, {X, Y, Z});
        BlockIterativeReconstructionOperator rec(rvol, views, projs.data(), p);
        rec.run();
        save(dir, "sart_volume.bin", rec.getReconstructedVolume().data(), rvol.voxelCount());
        std::printf("residual %.17g\n", rec.lastResidualSq());
        // weighted back projection of the same projections (the WBP plugin's algorithm)
        GPUMappedVolume wvol(fw, {X, Y, Z});
        WBP wbp(wvol, views, projs.data(),
                AlgebraicParameterSet::fromConfig(
                    {{"algorithm", "wbp"}, {"algorithm.numberOfIterations", "1"}, {"algorithm.lambda", "1.0"}}));
        wbp.run();
        save(dir, "wbp_volume.bin", wbp.getReconstructedVolume().data(), wvol.voxelCount());
        // blob basis functions: perspective views of a 24^3 phantom, blob SART from the
        // configuration keys with voxelisation of the result
        {
            const uint32_t B = 24, D = 32, BV = 4;
            std::vector<float> ph(B * B * B);
            for (uint32_t i = 0; i < ph.size(); ++i) ph[i] = (float)((i * 7 + (i / B) * 13) % 11) / 10.f;
            GPUMappedVolume pvol(fw, {B, B, B});
            pvol.upload(ph.data());
            etcu_view base{};
            const float pitch = 0.1f / (float)D;
            const float src[3] = {0.f, 0.f, -160.f}, det[3] = {-0.05f, -0.05f, -159.f};
            for (int i = 0; i < 3; ++i) {
                base.source[i] = src[i];
                base.detector[i] = det[i];
                base.hpitch[i] = i == 0 ? pitch : 0.f;
                base.vpitch[i] = i == 1 ? pitch : 0.f;
            }
            base.width = base.height = D;
            base.perspective = 1;
            std::vector<ScannerGeometry> bviews;
            std::vector<float> bprojs(BV * D * D);
            ForwardProjectionOperator bfp(pvol, BlobParameters::createDefault());
            for (uint32_t i = 0; i < BV; ++i) {
                bviews.push_back(ScannerGeometry(base).rotated(-45.f + 30.f * (float)i));
                bfp.setScannerGeometry(bviews.back());
                cuda(cudaMemset(dv, 0, D * D * 4));
                cuda(cudaMemset(dl, 0, D * D * 4));
                bfp.SetOutput(dv, dl);
                bfp.Execute(0);
                cuda(cudaMemcpy(bprojs.data() + i * D * D, dv, D * D * 4, cudaMemcpyDeviceToHost));
            }
            save(dir, "blob_projections.bin", bprojs.data(), bprojs.size());
            const AlgebraicParameterSet bp2 = AlgebraicParameterSet::fromConfig(
                {{"algorithm", "sart"}, {"algorithm.numberOfIterations", "1"}, {"algorithm.lambda", "0.5"},
                 {"optimization.projectionIteration", "identity"}, {"algorithm.basisFunctions", "blobs"},
                 {"output.options.enableVoxelization", "true"}});
            GPUMappedVolume bvol2(fw, {B, B, B});
            BlockIterativeReconstructionOperator brec(bvol2, bviews, bprojs.data(), bp2);
            brec.run();
            save(dir, "blob_coefficients.bin", bvol2.download().data(), bvol2.voxelCount());
            save(dir, "blob_voxels.bin", brec.getReconstructedVolume().data(), bvol2.voxelCount());
        }
        cudaFree(dv);
        cudaFree(dl);
        cudaFree(dr);
    } catch (const Exception& e) {
        std::printf("error %d %s\n", (int)e.status(), e.what());
        return 1;
    }
    return 0;
}
