// Device code of the learned warm start: a 3-level 3-D convolutional encoder-decoder
// (3x3x3 convolutions, 16 / 32 / 64 channels, BF16 storage, FP32 accumulation) whose
// forward, input-gradient and weight-gradient convolutions run on the 5th-generation
// tensor cores (tcgen05.mma, accumulators in tensor memory) with operand tiles brought
// into shared memory by the tensor memory accelerator (cp.async.bulk.tensor, local
// memory only, no cluster multicast).  The reference has no learned component; this
// is the warm start that feeds its `volume.initFile` entry
// (BlockIterativeConfiguration.cpp:36-41).
//
// Activation layout ("NC8"): bf16 [n * C/8 + c8][z][y][x][8]: every 8-channel chunk is a
// plane of 16-byte cells.  A tensor map of rank 5 {8, X, Y, Z, n*C/8} then delivers, for
// one output row of 128 voxels, the 130 x 3 x 3 halo of one or two chunks as planes of
// 16-byte rows, which is the tensor cores' K-major (and MN-major) layout without swizzle:
// eight rows of 16 bytes form one 128-byte core matrix, and the 27 taps of the 3x3x3
// stencil are 27 start addresses inside the same halo (+16 B per x step, +130*16 B per y
// step, +390*16 B per z step).  So one halo load feeds 27 MMAs.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace ws {

constexpr int kTileX = 128;                        // output voxels (MMA rows) per tile
constexpr int kHaloX = kTileX + 2;                 // halo width along x
constexpr uint32_t kHaloPlane = kHaloX * 9 * 16;   // one chunk of a 130 x 3 x 3 halo: 18,720 B
constexpr uint32_t kHaloBytes = 2 * kHaloPlane;    // two chunks = 16 channels = one MMA K step
constexpr uint64_t kWaitLimitNs = 1000000000ull;   // every wait gives up after 1 s

// Error word bits (sticky, read by the host after a call).
constexpr unsigned kErrWaitFull = 1u, kErrWaitEmpty = 2u, kErrWaitDone = 4u;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ uint64_t globaltimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// ---------------------------------------------------------------- mbarrier
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Waits for the phase with the given parity to complete; false after kWaitLimitNs.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = globaltimer();
    while (!mbar_try_wait(bar, parity))
        if (globaltimer() - t0 > kWaitLimitNs) return false;
    return true;
}

// ---------------------------------------------------------------- bulk copies (this GPU's memory only)
__device__ __forceinline__ void tma_load_5d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1, int c2,
                                            int c3, int c4) {
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, "
        "%6}], [%7];" ::"r"(smem_u32(dst)),
        "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_u32(bar))
        : "memory");
}
// 16-byte copy global -> shared; src_bytes 0 writes 16 zero bytes (no global read).
__device__ __forceinline__ void cp_async16z(uint32_t dst, const void* src, uint32_t src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit_group() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_group() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
// Generic-proxy shared-memory writes (cp.async) made visible to the async proxy (the
// tensor cores' operand reads).
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// ---------------------------------------------------------------- tensor memory and MMA
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {  // one full warp
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {  // one full warp
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// D (tensor memory) = A * B (+ D when accumulate != 0); bf16 operands from shared memory.
__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}
// Arrives on `bar` once every MMA this thread issued before has completed.
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}
// 16 consecutive 32-bit columns of this thread's lane (one full warp).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Shared-memory matrix descriptor, no swizzle (canonical "interleaved" layout: 8 rows of
// 16 bytes form a core matrix).  lbo / sbo in bytes: for K-major operands lbo is the step
// between the two 8-element K halves of an MMA and sbo the step between groups of 8 rows;
// for MN-major operands sbo is the step between groups of 8 M/N elements and lbo the step
// between groups of 8 K rows.  Bits 46-47 hold the descriptor version (1).
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// Instruction descriptor of kind::f16: bf16 A and B, FP32 accumulator, M x N, K-major (0)
// or MN-major (1) operands.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, int a_mn, int b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
           ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&h);
}
__device__ __forceinline__ void unpack_bf16x8(uint4 u, float (&v)[8]) {
    const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        float2 f = __bfloat1622float2(h[i]);
        v[2 * i] = f.x;
        v[2 * i + 1] = f.y;
    }
}

// ---------------------------------------------------------------- forward / input-gradient convolution
struct ConvDst {
    __nv_bfloat16* ptr;         // NC8 tensor of `channels` channels
    const __nv_bfloat16* mask;  // NULL, or an NC8 tensor of the same shape: values where mask <= 0 become 0
    int channels;
};

struct ConvArgs {
    int X, Y, Z, batch;    // voxel grid of input and output (same-size convolution)
    int nsteps;            // K steps of 16 channels over both sources
    int nkp0;              // steps from source 0 (the rest from source 1)
    int c8_0, c8_1;        // chunks per batch item of source 0 / 1 (dim-4 coordinate n * c8 + 2 kp)
    const __nv_bfloat16* p0;  // the sources as NC8 tensors (cp.async loaders)
    const __nv_bfloat16* p1;
    const __nv_bfloat16* w;  // [step][27 taps][2 halves][N][8] bf16
    int resident;          // 1: all steps' weights are loaded once into shared memory
    const float* bias;     // N values or NULL
    int relu;
    int head;              // 1: channel 0 only, out_f32 = in_f32 + scale * (acc + bias)
    ConvDst dst0, dst1;    // channels [0, n0) -> dst0, [n0, N) -> dst1
    int n0;
    const float* head_in;
    float* head_out;
    float head_scale;
    int stages;
    unsigned* err;
};

template <int N, int TY>
struct ConvShape {
    static constexpr uint32_t kHalo = (uint32_t)kHaloX * (TY + 2) * 3u * 16u * 2u;  // two chunks
    static constexpr uint32_t kPlane = (uint32_t)kHaloX * (TY + 2) * 3u * 16u;      // one chunk
    static constexpr uint32_t kW = 27u * 2u * N * 16u;                               // one step's weights
    static constexpr uint32_t kAcc = (uint32_t)TY * N;                               // columns per accumulator
    static constexpr uint32_t kCols = 2 * kAcc <= 32 ? 32 : 2 * kAcc <= 64 ? 64 : 2 * kAcc <= 128 ? 128
                                      : 2 * kAcc <= 256 ? 256 : 512;
    static_assert(2 * kAcc <= 512, "two accumulators must fit in tensor memory");
};

// Persistent convolution: a CTA takes tiles of 128 x-voxels by TY y-rows (one z, one batch
// item) round-robin.  Warp 0 streams the 130 x (TY + 2) x 3 halo of every 16-channel step
// (and, unless the weights are resident, the step's weights) through a ring of `stages`
// buffers; warp 1 issues 27 x TY MMAs per step into one of two tensor-memory accumulators;
// warps 2-5 drain the other accumulator (bias, ReLU, mask, BF16 store) meanwhile.
// kLoad 0 (default): warp 0 brings every halo with one tensor copy (cp.async.bulk.tensor);
// kLoad 1: warps 0-3 copy it with 16-byte cp.async (rows of 512 bytes per warp
// instruction), the MMA and epilogue warps follow.  The autotuner times both (on B200 the
// tensor copy was 1.6x faster on every layer of the 256 x 256 x 128 network).
template <int kLoad>
constexpr int conv_threads() { return kLoad ? 288 : 192; }

template <int N, int TY, int kLoad>
__global__ void __launch_bounds__(conv_threads<kLoad>(), 1) conv_tc_kernel(const __grid_constant__ CUtensorMap src0,
                                                                          const __grid_constant__ CUtensorMap src1,
                                                                          ConvArgs a) {
    using SH = ConvShape<N, TY>;
    static_assert(N % 16 == 0 && N >= 16 && N <= 256, "M = 128 needs N a multiple of 16");
    constexpr uint32_t kIdesc = idesc_bf16(128, N, 0, 0);
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    const int S = a.stages;
    const uint32_t wres = a.resident ? (uint32_t)a.nsteps * SH::kW : 0u;           // resident weights
    const uint32_t stage = (SH::kHalo + (a.resident ? 0u : SH::kW) + 1023u) & ~1023u;
    uint8_t* wsm = smem;                                                             // resident weights
    uint8_t* ring = smem + ((wres + 1023u) & ~1023u);
    uint64_t* full = (uint64_t*)(ring + (size_t)S * stage);
    uint64_t* empty = full + S;
    uint64_t* accf = empty + S;  // [2] accumulator written (MMA -> epilogue)
    uint64_t* acce = accf + 2;   // [2] accumulator drained (epilogue -> MMA)
    uint64_t* wbar = acce + 2;
    uint32_t* tmem_slot = (uint32_t*)(wbar + 1);

    const int ntx = (a.X + kTileX - 1) / kTileX;
    const int nty = (a.Y + TY - 1) / TY;
    const int ntiles = ntx * nty * a.Z * a.batch;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    constexpr int kLoaders = kLoad ? 128 : 1;        // arrivals that complete a stage
    constexpr int kMmaWarp = kLoad ? 4 : 1, kEpiWarp = kLoad ? 5 : 2;

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&full[s], kLoaders);
            mbar_init(&empty[s], 1);
        }
        for (int i = 0; i < 2; ++i) {
            mbar_init(&accf[i], 1);
            mbar_init(&acce[i], 4);
        }
        mbar_init(wbar, 1);
        mbar_fence_init();
    }
    if (warp == 0) tmem_alloc(tmem_slot, SH::kCols);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (kLoad && warp < 4) {
        // cp.async loaders: stage q's copies are issued, then stage q - (S - 1)'s are
        // waited for, fenced for the tensor cores and announced
        const int tid = threadIdx.x;
        if (tid == 0 && a.resident) {
            mbar_expect_tx(wbar, wres);
            bulk_load(wsm, a.w, wres, wbar);
        }
        constexpr int kRows = 2 * 3 * (TY + 2);
        constexpr int kElems = kRows * kHaloX;
        int q = 0;
        bool ok = true;
        auto announce = [&](int k) {  // stage of load k is in shared memory
            fence_proxy_async_smem();
            mbar_arrive(&full[k % S]);
        };
        auto drain_to = [&](int pending) {  // wait until at most `pending` groups are in flight
            switch (pending) {
            case 0: cp_async_wait_group<0>(); break;
            case 1: cp_async_wait_group<1>(); break;
            case 2: cp_async_wait_group<2>(); break;
            default: cp_async_wait_group<3>(); break;
            }
        };
        for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
            int t = tile;
            const int xt = t % ntx;
            t /= ntx;
            const int yt = t % nty;
            t /= nty;
            const int z = t % a.Z;
            const int n = t / a.Z;
            for (int s = 0; s < a.nsteps; ++s, ++q) {
                const int st = q % S;
                if (q >= S && !mbar_wait(&empty[st], ((q / S) - 1) & 1)) {
                    if (tid == 0) atomicOr(a.err, kErrWaitEmpty);
                    ok = false;
                    break;
                }
                const uint32_t halo = smem_u32(ring + (size_t)st * stage);
                const bool second = s >= a.nkp0;
                const int kp = second ? s - a.nkp0 : s;
                const __nv_bfloat16* src = second ? a.p1 : a.p0;
                const int cbase = n * (second ? a.c8_1 : a.c8_0) + 2 * kp;
                for (int e = tid; e < kElems; e += 128) {
                    const int row = e / kHaloX, xi = e - row * kHaloX;
                    const int c = row / (3 * (TY + 2)), rem = row - c * (3 * (TY + 2));
                    const int dz = rem / (TY + 2), dy = rem - dz * (TY + 2);
                    const int xx = xt * kTileX - 1 + xi, yy = yt * TY - 1 + dy, zz = z - 1 + dz;
                    const bool in = xx >= 0 && xx < a.X && yy >= 0 && yy < a.Y && zz >= 0 && zz < a.Z;
                    const __nv_bfloat16* g =
                        in ? src + ((((size_t)(cbase + c) * a.Z + zz) * a.Y + yy) * a.X + xx) * 8 : src;
                    cp_async16z(halo + (uint32_t)e * 16u, g, in ? 16u : 0u);
                }
                if (!a.resident) {
                    const __nv_bfloat16* wsrc = a.w + (size_t)s * (SH::kW / 2);
                    for (int e = tid; e < (int)(SH::kW / 16); e += 128)
                        cp_async16z(halo + SH::kHalo + (uint32_t)e * 16u, wsrc + (size_t)e * 8, 16u);
                }
                cp_async_commit_group();
                if (q >= S - 1) {
                    drain_to(S - 1);
                    announce(q - (S - 1));
                }
            }
        }
        // the last stages: announce what this thread issued and has not announced yet
        const int first_open = q - (S - 1) < 0 ? 0 : q - (S - 1);
        cp_async_wait_group<0>();
        for (int k = first_open; k < q; ++k) announce(k);
    } else if (!kLoad && warp == 0) {
        if (lane == 0) {
            if (a.resident) {
                mbar_expect_tx(wbar, wres);
                bulk_load(wsm, a.w, wres, wbar);
            }
            int q = 0;
            bool ok = true;
            for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
                int t = tile;
                const int xt = t % ntx;
                t /= ntx;
                const int yt = t % nty;
                t /= nty;
                const int z = t % a.Z;
                const int n = t / a.Z;
                for (int s = 0; s < a.nsteps; ++s, ++q) {
                    const int st = q % S;
                    if (q >= S && !mbar_wait(&empty[st], ((q / S) - 1) & 1)) {
                        atomicOr(a.err, kErrWaitEmpty);
                        ok = false;
                        break;
                    }
                    uint8_t* halo = ring + (size_t)st * stage;
                    mbar_expect_tx(&full[st], SH::kHalo + (a.resident ? 0u : SH::kW));
                    const bool second = s >= a.nkp0;
                    const int kp = second ? s - a.nkp0 : s;
                    const int c4 = n * (second ? a.c8_1 : a.c8_0) + 2 * kp;
                    tma_load_5d(halo, second ? &src1 : &src0, &full[st], 0, xt * kTileX - 1, yt * TY - 1, z - 1, c4);
                    if (!a.resident)
                        bulk_load(halo + SH::kHalo, a.w + (size_t)s * (SH::kW / 2), SH::kW, &full[st]);
                }
            }
        }
    } else if (warp == kMmaWarp) {
        if (lane == 0) {
            bool ok = !a.resident || mbar_wait(wbar, 0);
            if (!ok) atomicOr(a.err, kErrWaitFull);
            int q = 0, i = 0;
            for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x, ++i) {
                const int acc = i & 1;
                if (i >= 2 && !mbar_wait(&acce[acc], ((i >> 1) - 1) & 1)) {
                    atomicOr(a.err, kErrWaitEmpty);
                    break;
                }
                tc_fence_after();
                const uint32_t dacc = tmem + (uint32_t)acc * SH::kAcc;
                for (int s = 0; s < a.nsteps; ++s, ++q) {
                    const int st = q % S;
                    if (!mbar_wait(&full[st], (q / S) & 1)) {
                        atomicOr(a.err, kErrWaitFull);
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t hbase = smem_u32(ring + (size_t)st * stage);
                    const uint32_t wbase = a.resident ? smem_u32(wsm) + (uint32_t)s * SH::kW : hbase + SH::kHalo;
                    // per-tap descriptors as the base descriptor plus a constant (address / 16
                    // in the start-address field; shared-memory addresses stay below 256 KiB)
                    const uint64_t a0 = sdesc(hbase, SH::kPlane, 128);
                    const uint64_t b0 = sdesc(wbase, N * 16u, 128);
#pragma unroll
                    for (int tap = 0; tap < 27; ++tap) {
                        const int dz = tap / 9, dy = (tap / 3) % 3, dx = tap % 3;
                        const uint64_t bd = b0 + (uint64_t)((tap * 2u * N * 16u) >> 4);
#pragma unroll
                        for (int ty = 0; ty < TY; ++ty) {
                            const uint32_t aoff = (uint32_t)(((dz * (TY + 2) + ty + dy) * kHaloX + dx) * 16);
                            umma_bf16(dacc + (uint32_t)(ty * N), a0 + (uint64_t)(aoff >> 4), bd, kIdesc,
                                      (s > 0 || tap > 0) ? 1u : 0u);
                        }
                    }
                    umma_commit(&empty[st]);
                }
                if (!ok) break;
                umma_commit(&accf[acc]);
            }
        }
    } else if (warp >= kEpiWarp) {
        // epilogue: warp quarter (warp % 4) reads tensor-memory lanes 32 * (warp % 4) ...
        const int quarter = warp & 3;
        const int m = quarter * 32 + lane;
        const size_t plane = (size_t)a.Z * a.Y * a.X;
        int i = 0;
        for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++i) {
            const int acc = i & 1;
            const bool got = mbar_wait(&accf[acc], (i >> 1) & 1);
            __syncwarp();
            if (!got) {
                if (lane == 0) atomicOr(a.err, kErrWaitDone);
                break;
            }
            tc_fence_after();
            int t = tile;
            const int xt = t % ntx;
            t /= ntx;
            const int yt = t % nty;
            t /= nty;
            const int z = t % a.Z;
            const int n = t / a.Z;
            const int x = xt * kTileX + m;
            const uint32_t dacc = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)acc * SH::kAcc;
#pragma unroll 1
            for (int ty = 0; ty < TY; ++ty) {
                const int y = yt * TY + ty;
                const bool valid = x < a.X && y < a.Y;
                const size_t vox = ((size_t)z * a.Y + y) * a.X + x;
                if (a.head) {
                    uint32_t r[16];
                    tmem_ld16(dacc + (uint32_t)(ty * N), r);
                    tmem_wait_ld();
                    if (valid) {
                        const size_t idx = (size_t)n * plane + vox;
                        const float accv = __uint_as_float(r[0]) + (a.bias ? a.bias[0] : 0.f);
                        a.head_out[idx] = fmaf(a.head_scale, accv, a.head_in[idx]);
                    }
                    continue;
                }
#pragma unroll
                for (int c = 0; c < N / 16; ++c) {
                    uint32_t r[16];
                    tmem_ld16(dacc + (uint32_t)(ty * N + c * 16), r);
                    tmem_wait_ld();
                    if (!valid) continue;
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int ch = c * 16 + h * 8;
                        float v[8];
#pragma unroll
                        for (int j = 0; j < 8; ++j) {
                            v[j] = __uint_as_float(r[h * 8 + j]);
                            if (a.bias) v[j] += a.bias[ch + j];
                            if (a.relu) v[j] = fmaxf(v[j], 0.f);
                        }
                        const bool first = ch < a.n0;
                        const ConvDst& d = first ? a.dst0 : a.dst1;
                        const int c8 = (first ? ch : ch - a.n0) >> 3;
                        const size_t off = ((size_t)(n * (d.channels >> 3) + c8) * plane + vox) * 8;
                        if (d.mask) {
                            float mk[8];
                            unpack_bf16x8(*reinterpret_cast<const uint4*>(d.mask + off), mk);
#pragma unroll
                            for (int j = 0; j < 8; ++j) v[j] = mk[j] > 0.f ? v[j] : 0.f;
                        }
                        uint4 o;
                        o.x = pack_bf16x2(v[0], v[1]);
                        o.y = pack_bf16x2(v[2], v[3]);
                        o.z = pack_bf16x2(v[4], v[5]);
                        o.w = pack_bf16x2(v[6], v[7]);
                        *reinterpret_cast<uint4*>(d.ptr + off) = o;
                    }
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&acce[acc]);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, SH::kCols);
    }
}

// ---------------------------------------------------------------- z-streamed convolution, 16 outputs
// For the 16-output-channel layers the MMAs above are N = 16 wide and re-read their 128-row
// A operand from shared memory for each of the 27 taps.  Here a CTA walks a column of
// tiles (128 x-voxels by TY y-rows) along z, one input z slice at a time, and folds the
// three dz taps into N: for input slice zi and tap (dy, dx) one MMA of N = 48 computes
// D[zi][g][o] = sum_{c, dy, dx} W[dz = g - 1][dy][dx][c][o] * In[zi][y + dy - 1][x + dx - 1][c]
// for g = 0, 1, 2, and the epilogue forms out[z] = D[z - 1][0] + D[z][1] + D[z + 1][2]
// (the 3x3x3 convolution; zero slices outside the volume come from the tensor copy's
// out-of-range fill).  So 9 MMAs per K step and row instead of 27, and a 1-slice halo
// instead of 3.  Slice j of a segment (zi = z0 - 1 + j) accumulates in tensor-memory slot
// (global slice count) % 4 of TY x 48 columns; the epilogue of output z0 + j - 2 (after
// slice j) reads slots of j - 2, j - 1, j and releases j - 2's (all three at the
// segment's last output), so the MMAs run up to two slices ahead of the epilogue.
template <int NOUT, int TY>
struct ZfoldShape {
    static constexpr uint32_t kN = 3u * NOUT;                              // MMA N: three dz groups
    static constexpr uint32_t kPlane = (uint32_t)kHaloX * (TY + 2) * 16u;  // one 8-channel chunk, one z
    static constexpr uint32_t kHalo = 2u * kPlane;                         // 16 channels = one K step
    static constexpr uint32_t kW = 9u * 2u * kN * 16u;                     // one step's weights
    static constexpr uint32_t kSlot = (uint32_t)TY * kN;                   // tensor-memory columns per slice
    static_assert(4 * kSlot <= 512, "four slices must fit in tensor memory");
};

struct ZfoldArgs {
    int X, Y, Z, batch;
    int zseg;              // output z slices per work unit
    int nsteps, nkp0, c8_0, c8_1;
    const __nv_bfloat16* w;  // [step][9 taps (dy, dx)][2 halves][3 dz x NOUT][8] bf16
    int resident;
    const float* bias;     // NOUT values
    int relu;
    ConvDst dst;           // NOUT channels
    int head;              // 1: channel 0 only, head_out = head_in + head_scale * (acc + bias) (FP32)
    const float* head_in;
    float* head_out;
    float head_scale;
    int stages;
    unsigned* err;
};

constexpr int kZfoldThreads = 320;  // warp 0 loads, warp 1 issues the MMAs, warps 2-9 drain

template <int NOUT, int TY>
__global__ void __launch_bounds__(kZfoldThreads, 1) conv_zfold_kernel(const __grid_constant__ CUtensorMap src0,
                                                            const __grid_constant__ CUtensorMap src1, ZfoldArgs a) {
    using SH = ZfoldShape<NOUT, TY>;
    constexpr uint32_t kIdesc = idesc_bf16(128, SH::kN, 0, 0);
    constexpr uint32_t kCols = 512;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    const int S = a.stages;
    const uint32_t wres = a.resident ? (uint32_t)a.nsteps * SH::kW : 0u;
    const uint32_t stage = (SH::kHalo + (a.resident ? 0u : SH::kW) + 1023u) & ~1023u;
    uint8_t* wsm = smem;
    uint8_t* ring = smem + ((wres + 1023u) & ~1023u);
    uint64_t* full = (uint64_t*)(ring + (size_t)S * stage);
    uint64_t* empty = full + S;
    uint64_t* accf = empty + S;  // [4] slice written (MMA -> epilogue)
    uint64_t* acce = accf + 4;   // [4] slice released (epilogue -> MMA)
    uint64_t* wbar = acce + 4;
    uint32_t* tmem_slot = (uint32_t*)(wbar + 1);

    const int ntx = (a.X + kTileX - 1) / kTileX;
    const int nty = (a.Y + TY - 1) / TY;
    const int nseg = (a.Z + a.zseg - 1) / a.zseg;
    const int nunits = ntx * nty * nseg * a.batch;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    auto unit_of = [&](int u, int& xt, int& yt, int& z0, int& len, int& n) {
        xt = u % ntx;
        u /= ntx;
        yt = u % nty;
        u /= nty;
        const int sg = u % nseg;
        n = u / nseg;
        z0 = sg * a.zseg;
        len = min(a.zseg, a.Z - z0);
    };

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int i = 0; i < 4; ++i) {
            mbar_init(&accf[i], 1);
            mbar_init(&acce[i], 8);  // the eight epilogue warps
        }
        mbar_init(wbar, 1);
        mbar_fence_init();
    }
    if (warp == 0) tmem_alloc(tmem_slot, kCols);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            if (a.resident) {
                mbar_expect_tx(wbar, wres);
                bulk_load(wsm, a.w, wres, wbar);
            }
            int q = 0;
            bool ok = true;
            for (int u = blockIdx.x; u < nunits && ok; u += gridDim.x) {
                int xt, yt, z0, len, n;
                unit_of(u, xt, yt, z0, len, n);
                for (int j = 0; j < len + 2 && ok; ++j)
                    for (int s = 0; s < a.nsteps; ++s, ++q) {
                        const int st = q % S;
                        if (q >= S && !mbar_wait(&empty[st], ((q / S) - 1) & 1)) {
                            atomicOr(a.err, kErrWaitEmpty);
                            ok = false;
                            break;
                        }
                        uint8_t* halo = ring + (size_t)st * stage;
                        mbar_expect_tx(&full[st], SH::kHalo + (a.resident ? 0u : SH::kW));
                        const bool second = s >= a.nkp0;
                        const int kp = second ? s - a.nkp0 : s;
                        const int c4 = n * (second ? a.c8_1 : a.c8_0) + 2 * kp;
                        tma_load_5d(halo, second ? &src1 : &src0, &full[st], 0, xt * kTileX - 1, yt * TY - 1,
                                    z0 - 1 + j, c4);
                        if (!a.resident)
                            bulk_load(halo + SH::kHalo, a.w + (size_t)s * (SH::kW / 2), SH::kW, &full[st]);
                    }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            bool ok = !a.resident || mbar_wait(wbar, 0);
            if (!ok) atomicOr(a.err, kErrWaitFull);
            int q = 0, G = 0;
            for (int u = blockIdx.x; u < nunits && ok; u += gridDim.x) {
                int xt, yt, z0, len, n;
                unit_of(u, xt, yt, z0, len, n);
                for (int j = 0; j < len + 2 && ok; ++j, ++G) {
                    const int slot = G & 3;
                    if (G >= 4 && !mbar_wait(&acce[slot], ((G >> 2) - 1) & 1)) {
                        atomicOr(a.err, kErrWaitEmpty);
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t dslot = tmem + (uint32_t)slot * SH::kSlot;
                    for (int s = 0; s < a.nsteps; ++s, ++q) {
                        const int st = q % S;
                        if (!mbar_wait(&full[st], (q / S) & 1)) {
                            atomicOr(a.err, kErrWaitFull);
                            ok = false;
                            break;
                        }
                        tc_fence_after();
                        const uint32_t hbase = smem_u32(ring + (size_t)st * stage);
                        const uint32_t wbase =
                            a.resident ? smem_u32(wsm) + (uint32_t)s * SH::kW : hbase + SH::kHalo;
                        // one descriptor per operand base; every tap's is the base plus a constant
                        // (the start-address field is address / 16, and every address here is
                        // below 256 KiB, so the add never leaves the field)
                        const uint64_t a0 = sdesc(hbase, SH::kPlane, 128);
                        const uint64_t b0 = sdesc(wbase, SH::kN * 16u, 128);
#pragma unroll
                        for (int tap = 0; tap < 9; ++tap) {
                            const int dy = tap / 3, dx = tap % 3;
                            const uint64_t bd = b0 + (uint64_t)((tap * 2u * SH::kN * 16u) >> 4);
#pragma unroll
                            for (int ty = 0; ty < TY; ++ty) {
                                const uint32_t aoff = (uint32_t)(((ty + dy) * kHaloX + dx) * 16);
                                umma_bf16(dslot + (uint32_t)ty * SH::kN, a0 + (uint64_t)(aoff >> 4), bd, kIdesc,
                                          (s > 0 || tap > 0) ? 1u : 0u);
                            }
                        }
                        umma_commit(&empty[st]);
                    }
                    if (!ok) break;
                    umma_commit(&accf[slot]);
                }
            }
        }
    } else {
        // epilogue: warp quarter (warp % 4) reads tensor-memory lanes 32 * (warp % 4) ...;
        // two warps per quarter, one per tile row (TY = 2) or per 16 channels (TY = 1)
        const int quarter = warp & 3, part = (warp - 2) >> 2;
        const int m = quarter * 32 + lane;
        const size_t plane = (size_t)a.Z * a.Y * a.X;
        float bias[NOUT];
#pragma unroll
        for (int c = 0; c < NOUT; ++c) bias[c] = a.bias ? a.bias[c] : 0.f;
        int G = 0;
        bool ok = true;
        for (int u = blockIdx.x; u < nunits && ok; u += gridDim.x) {
            int xt, yt, z0, len, n;
            unit_of(u, xt, yt, z0, len, n);
            const int x = xt * kTileX + m;
            for (int j = 0; j < len + 2; ++j, ++G) {
                if (j < 2) continue;  // output z0 + j - 2 needs slices j - 2, j - 1, j
                const bool got = mbar_wait(&accf[G & 3], (G >> 2) & 1);
                __syncwarp();
                if (!got) {
                    if (lane == 0) atomicOr(a.err, kErrWaitDone);
                    ok = false;
                    break;
                }
                tc_fence_after();
                const int z = z0 + j - 2;
                const uint32_t lanes = (uint32_t)(quarter * 32) << 16;
                const uint32_t s0 = tmem + lanes + (uint32_t)((G - 2) & 3) * SH::kSlot;
                const uint32_t s1 = tmem + lanes + (uint32_t)((G - 1) & 3) * SH::kSlot;
                const uint32_t s2 = tmem + lanes + (uint32_t)(G & 3) * SH::kSlot;
#pragma unroll 1
                for (int ty = 0; ty < TY; ++ty) {
                    if (TY == 2 && ty != part) continue;
                    const int y = yt * TY + ty;
                    const bool valid = x < a.X && y < a.Y;
                    const size_t vox = ((size_t)z * a.Y + y) * a.X + x;
#pragma unroll
                    for (int c16 = 0; c16 < NOUT / 16; ++c16) {
                        if (TY == 1 && NOUT == 32 && c16 != part) continue;
                        const uint32_t col = (uint32_t)ty * SH::kN + (uint32_t)c16 * 16u;
                        uint32_t r0[16], r1[16], r2[16];
                        tmem_ld16(s0 + col, r0);             // dz = -1 of slice z - 1
                        tmem_ld16(s1 + col + NOUT, r1);      // dz = 0 of slice z
                        tmem_ld16(s2 + col + 2 * NOUT, r2);  // dz = +1 of slice z + 1
                        tmem_wait_ld();
                        if (!valid) continue;
                        if (a.head) {
                            const size_t idx = (size_t)n * plane + vox;
                            const float accv =
                                __uint_as_float(r0[0]) + __uint_as_float(r1[0]) + __uint_as_float(r2[0]) + bias[0];
                            a.head_out[idx] = fmaf(a.head_scale, accv, a.head_in[idx]);
                            continue;
                        }
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            float v[8];
#pragma unroll
                            for (int k = 0; k < 8; ++k) {
                                const int c = h * 8 + k;
                                v[k] = __uint_as_float(r0[c]) + __uint_as_float(r1[c]) + __uint_as_float(r2[c]);
                                v[k] += bias[c16 * 16 + c];
                                if (a.relu) v[k] = fmaxf(v[k], 0.f);
                            }
                            const size_t off =
                                ((size_t)(n * (a.dst.channels >> 3) + c16 * 2 + h) * plane + vox) * 8;
                            if (a.dst.mask) {
                                float mk[8];
                                unpack_bf16x8(*reinterpret_cast<const uint4*>(a.dst.mask + off), mk);
#pragma unroll
                                for (int k = 0; k < 8; ++k) v[k] = mk[k] > 0.f ? v[k] : 0.f;
                            }
                            uint4 o;
                            o.x = pack_bf16x2(v[0], v[1]);
                            o.y = pack_bf16x2(v[2], v[3]);
                            o.z = pack_bf16x2(v[4], v[5]);
                            o.w = pack_bf16x2(v[6], v[7]);
                            *reinterpret_cast<uint4*>(a.dst.ptr + off) = o;
                        }
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) {
                    mbar_arrive(&acce[(G - 2) & 3]);  // slice j - 2 is no longer needed
                    if (j == len + 1) {               // the segment's last output: its last two slices too
                        mbar_arrive(&acce[(G - 1) & 3]);
                        mbar_arrive(&acce[G & 3]);
                    }
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, kCols);
    }
}

// Forward weights of an nout-output layer for conv_zfold_kernel: [step][tap9 = dy * 3 + dx]
// [half][r = g * nout + o][8] = W[tap = g * 9 + tap9][o][ci] (input z offset g - 1), bf16,
// zero past cout / cin.
__global__ void relayout_zfold_kernel(const float* __restrict__ W, int cout, int cin_total, int nout, int nsteps,
                                      __nv_bfloat16* __restrict__ out) {
    const int nn = 3 * nout;
    const int total = nsteps * 9 * 2 * nn * 8;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    int t = i;
    const int j = t % 8;
    t /= 8;
    const int r = t % nn;
    t /= nn;
    const int half = t % 2;
    t /= 2;
    const int tap9 = t % 9;
    const int step = t / 9;
    const int g = r / nout, o = r % nout;
    const int tap = g * 9 + tap9;
    const int ci = step * 16 + half * 8 + j;
    const float w = (o < cout && ci < cin_total) ? W[((size_t)tap * cout + o) * cin_total + ci] : 0.f;
    out[i] = __float2bfloat16_rn(w);
}

// ---------------------------------------------------------------- weight gradient
// dW[tap][co][ci] = sum over voxels v of dPre[v][co] * In[v + off(tap)][ci].  Per tile of
// 128 voxels the K dimension of the MMA runs over voxels: A = dPre^T (M = co, padded to
// 128 rows, MN-major: 8 channels contiguous per voxel row), B = the tap-shifted input
// (N = ci, MN-major), D[co][ci] of every tap of the CTA's tap group accumulates in tensor
// memory over all tiles the CTA takes.
struct WgradArgs {
    int X, Y, Z, batch;
    int in_c8;             // chunks per batch item of the input tensor
    int out_c8;            // chunks per batch item of dPre (COUT / 8)
    int cout;              // real output channels (rows of D that are written)
    int group_mode;        // 0: all 27 taps, box 130x3x3; 1: one dz (9 taps), box 130x3x1; 2: one (dz, dy), box 130x1x1
    int ranges;            // CTAs per tap group (voxel tiles are dealt round-robin)
    float* partial;        // [ranges][27][cout][CIN]
    int stages;
    unsigned* err;
};

template <int CIN>
__global__ void __launch_bounds__(128) wgrad_tc_kernel(const __grid_constant__ CUtensorMap in_map,
                                                       const __grid_constant__ CUtensorMap dpre_map, WgradArgs a) {
    static_assert(CIN == 16 || CIN == 32 || CIN == 64, "input chunks of 16, 32 or 64 channels");
    constexpr uint32_t kA = 16u * kTileX * 16u;  // dPre: 16 planes of 128 voxel rows (M = 128)
    constexpr uint32_t kIdesc = idesc_bf16(128, CIN, 1, 1);
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    const int mode = a.group_mode;
    const int ny = mode == 2 ? 1 : 3, nz = mode == 0 ? 3 : 1;
    const int ntaps = mode == 0 ? 27 : (mode == 1 ? 9 : 3);
    const uint32_t bplane = (uint32_t)kHaloX * ny * nz * 16u;
    const uint32_t bbytes = bplane * (CIN / 8);
    const uint32_t stage = (kA + bbytes + 1023u) & ~1023u;
    const int S = a.stages;
    uint64_t* full = (uint64_t*)(smem + S * stage);
    uint64_t* empty = full + S;
    uint64_t* done = empty + S;
    uint32_t* tmem_slot = (uint32_t*)(done + 1);
    const uint32_t cols_needed = (uint32_t)ntaps * CIN;
    const uint32_t ncols = cols_needed <= 32 ? 32 : cols_needed <= 64 ? 64 : cols_needed <= 128 ? 128
                           : cols_needed <= 256 ? 256 : 512;

    const int ngroups = mode == 0 ? 1 : (mode == 1 ? 3 : 9);
    const int g = blockIdx.x % ngroups;
    const int r = blockIdx.x / ngroups;
    const int gdz = mode == 2 ? g / 3 : g;  // dz of the group (modes 1, 2)
    const int gdy = mode == 2 ? g % 3 : 0;  // dy of the group (mode 2)
    const int ntx = (a.X + kTileX - 1) / kTileX;
    const int ntiles = ntx * a.Y * a.Z * a.batch;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(done, 1);
        mbar_fence_init();
    }
    if (warp == 0) tmem_alloc(tmem_slot, ncols);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const uint32_t abytes = (uint32_t)a.out_c8 * kTileX * 16u;

    if (warp == 0 && lane == 0) {
        int i = 0;
        for (int tile = r; tile < ntiles; tile += a.ranges, ++i) {
            const int st = i % S;
            if (i >= S && !mbar_wait(&empty[st], ((i / S) - 1) & 1)) {
                atomicOr(a.err, kErrWaitEmpty);
                break;
            }
            int t = tile;
            const int xt = t % ntx;
            t /= ntx;
            const int y = t % a.Y;
            t /= a.Y;
            const int z = t % a.Z;
            const int n = t / a.Z;
            uint8_t* sa = smem + st * stage;
            mbar_expect_tx(&full[st], abytes + bbytes);
            tma_load_5d(sa, &dpre_map, &full[st], 0, xt * kTileX, y, z, n * a.out_c8);
            const int by = mode == 2 ? y - 1 + gdy : y - 1;
            const int bz = mode == 0 ? z - 1 : z - 1 + gdz;
            tma_load_5d(sa + kA, &in_map, &full[st], 0, xt * kTileX - 1, by, bz, n * a.in_c8);
        }
    } else if (warp == 1 && lane == 0) {
        int i = 0;
        bool ok = true;
        for (int tile = r; tile < ntiles; tile += a.ranges, ++i) {
            const int st = i % S;
            if (!mbar_wait(&full[st], (i / S) & 1)) {
                atomicOr(a.err, kErrWaitFull);
                ok = false;
                break;
            }
            tc_fence_after();
            const uint32_t abase = smem_u32(smem + st * stage);
            const uint32_t bbase = abase + kA;
#pragma unroll 1
            for (int j = 0; j < ntaps; ++j) {
                int dz, dy, dx;
                if (mode == 0) { dz = j / 9; dy = (j / 3) % 3; dx = j % 3; }
                else if (mode == 1) { dz = 0; dy = j / 3; dx = j % 3; }
                else { dz = 0; dy = 0; dx = j; }
                const uint32_t boff = (uint32_t)(((dz * ny + dy) * kHaloX + dx) * 16);
#pragma unroll
                for (int k = 0; k < kTileX / 16; ++k) {
                    const uint64_t ad = sdesc(abase + k * 256u, 128, kTileX * 16u);
                    const uint64_t bd = sdesc(bbase + boff + k * 256u, 128, bplane);
                    umma_bf16(tmem + (uint32_t)(j * CIN), ad, bd, kIdesc, (i > 0 || k > 0) ? 1u : 0u);
                }
            }
            umma_commit(&empty[st]);
        }
        if (ok) umma_commit(done);
    }
    __syncwarp();
    const bool got = mbar_wait(done, 0);
    if (!got && threadIdx.x == 0) atomicOr(a.err, kErrWaitDone);
    __syncwarp();
    tc_fence_after();
    if (got && warp * 32 < a.cout) {
        // lane = output channel co; columns j * CIN + ci
        const int co = warp * 32 + lane;
        const int tap_base = mode == 0 ? 0 : (mode == 1 ? gdz * 9 : gdz * 9 + gdy * 3);
        for (int j = 0; j < ntaps; ++j) {
#pragma unroll
            for (int c = 0; c < CIN / 16; ++c) {
                uint32_t v[16];
                tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(j * CIN + c * 16), v);
                tmem_wait_ld();
                if (co < a.cout) {
                    float* dst = a.partial + (((size_t)r * 27 + tap_base + j) * a.cout + co) * CIN + c * 16;
#pragma unroll
                    for (int q = 0; q < 16; q += 4)
                        *reinterpret_cast<float4*>(dst + q) = make_float4(
                            __uint_as_float(v[q]), __uint_as_float(v[q + 1]), __uint_as_float(v[q + 2]),
                            __uint_as_float(v[q + 3]));
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, ncols);
    }
}

// ---------------------------------------------------------------- CUDA-core helpers
// grad[t][co][ci_off + ci] (row length cin_total) = sum over ranges of
// partial[r][t][co][ci] (row length cin), for ci < cin_used.
__global__ void wgrad_reduce_kernel(const float* __restrict__ partial, int ranges, int cout, int cin, int cin_used,
                                    float* __restrict__ grad, int cin_total, int ci_off) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = 27 * cout * cin_used;
    if (i >= n) return;
    const int ci = i % cin_used;
    const int tc = i / cin_used;  // t * cout + co
    const size_t stride = (size_t)27 * cout * cin;
    float s = 0.f;
    for (int r = 0; r < ranges; ++r) s += partial[(size_t)r * stride + (size_t)tc * cin + ci];
    grad[(size_t)tc * cin_total + ci_off + ci] = s;
}

// db[c] += sum over voxels of an NC8 tensor's channel c (batch items included).
__global__ void channel_sum_kernel(const __nv_bfloat16* __restrict__ t, int c8, int batch, size_t plane,
                                   int cout, float* __restrict__ db) {
    // blockIdx.y = chunk; blockIdx.x strides the (batch, voxel) range
    const int chunk = blockIdx.y;
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const size_t total = (size_t)batch * plane;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const size_t n = i / plane, v = i % plane;
        float f[8];
        unpack_bf16x8(*reinterpret_cast<const uint4*>(t + ((n * c8 + chunk) * plane + v) * 8), f);
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[j] += f[j];
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        float s = acc[j];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if ((threadIdx.x & 31) == 0 && chunk * 8 + j < cout) atomicAdd(&db[chunk * 8 + j], s);
    }
}

// First layer and head (one input / one output channel: no GEMM shape) on the CUDA
// cores.  A block of 256 threads computes a 32 x 8 tile of output voxels at one z; the
// 34 x 10 x 3 input halo is staged in shared memory first.  Weights rounded to BF16 as
// the tensor path holds them, FP32 accumulation.
constexpr int kEndTx = 32, kEndTy = 8, kEndHx = kEndTx + 2, kEndHy = kEndTy + 2;
constexpr int kEndHalo = kEndHx * kEndHy * 3;

// e1a[co] = relu(b[co] + sum_t x(v + off(t)) W[t][co]), x = bf16(v / scale); 16 output
// channels stored as the two chunks of an NC8 tensor.  W: FP32 master [27][16].
// Grid: (ceil(X / 32), ceil(Y / 8), Z * batch).
__global__ void __launch_bounds__(256) conv_in_kernel(const float* __restrict__ vin, float inv_scale, int X, int Y,
                                                       int Z, int batch, const float* __restrict__ W,
                                                       const float* __restrict__ bias, __nv_bfloat16* __restrict__ out) {
    __shared__ __align__(16) float ws_[27 * 16];
    __shared__ float bs_[16];
    __shared__ float halo[kEndHalo];
    const int tid = threadIdx.x;
    for (int i = tid; i < 27 * 16; i += 256) ws_[i] = __bfloat162float(__float2bfloat16_rn(W[i]));
    if (tid < 16) bs_[tid] = bias[tid];
    const int x0 = blockIdx.x * kEndTx, y0 = blockIdx.y * kEndTy;
    const int z = blockIdx.z % Z, n = blockIdx.z / Z;
    const size_t plane = (size_t)X * Y * Z;
    const float* src = vin + (size_t)n * plane;
    for (int i = tid; i < kEndHalo; i += 256) {
        const int hx = i % kEndHx, hy = (i / kEndHx) % kEndHy, hz = i / (kEndHx * kEndHy);
        const int xx = x0 - 1 + hx, yy = y0 - 1 + hy, zz = z - 1 + hz;
        float v = 0.f;
        if (xx >= 0 && xx < X && yy >= 0 && yy < Y && zz >= 0 && zz < Z)
            v = __bfloat162float(__float2bfloat16_rn(src[((size_t)zz * Y + yy) * X + xx] * inv_scale));
        halo[i] = v;
    }
    __syncthreads();
    const int tx = tid % kEndTx, ty = tid / kEndTx;
    const int x = x0 + tx, y = y0 + ty;
    if (x >= X || y >= Y) return;
    // the 16 channels as 8 pairs: one paired FMA per pair (each lane the fmaf of one channel)
    float2 acc2[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) acc2[c] = make_float2(bs_[2 * c], bs_[2 * c + 1]);
    const float2* w2 = reinterpret_cast<const float2*>(ws_);
#pragma unroll
    for (int t = 0; t < 27; ++t) {
        const float xv = halo[((t / 9) * kEndHy + ty + (t / 3) % 3) * kEndHx + tx + t % 3];
        const float2 xx = make_float2(xv, xv);
#pragma unroll
        for (int c = 0; c < 8; ++c) acc2[c] = __ffma2_rn(xx, w2[t * 8 + c], acc2[c]);
    }
    float acc[16];
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        acc[2 * c] = acc2[c].x;
        acc[2 * c + 1] = acc2[c].y;
    }
    const size_t v = ((size_t)z * Y + y) * X + x;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        uint4 o;
        o.x = pack_bf16x2(fmaxf(acc[8 * h + 0], 0.f), fmaxf(acc[8 * h + 1], 0.f));
        o.y = pack_bf16x2(fmaxf(acc[8 * h + 2], 0.f), fmaxf(acc[8 * h + 3], 0.f));
        o.z = pack_bf16x2(fmaxf(acc[8 * h + 4], 0.f), fmaxf(acc[8 * h + 5], 0.f));
        o.w = pack_bf16x2(fmaxf(acc[8 * h + 6], 0.f), fmaxf(acc[8 * h + 7], 0.f));
        *reinterpret_cast<uint4*>(out + (((size_t)n * 2 + h) * plane + v) * 8) = o;
    }
}

// out = vin + scale * (b + sum_t sum_ci d1b(v + off(t))[ci] W[t][ci]) from a 16-channel NC8
// tensor.  W: FP32 master [27][1][16].  Grid as conv_in_kernel.
__global__ void __launch_bounds__(256) conv_head_kernel(const __nv_bfloat16* __restrict__ in, int X, int Y, int Z,
                                                         int batch, const float* __restrict__ W,
                                                         const float* __restrict__ bias,
                                                         const float* __restrict__ vin, float scale,
                                                         float* __restrict__ out) {
    __shared__ float ws_[27 * 16];
    __shared__ __align__(16) uint4 halo[2][kEndHalo];  // the two 8-channel chunks
    const int tid = threadIdx.x;
    for (int i = tid; i < 27 * 16; i += 256) ws_[i] = __bfloat162float(__float2bfloat16_rn(W[i]));
    const int x0 = blockIdx.x * kEndTx, y0 = blockIdx.y * kEndTy;
    const int z = blockIdx.z % Z, n = blockIdx.z / Z;
    const size_t plane = (size_t)X * Y * Z;
    for (int i = tid; i < 2 * kEndHalo; i += 256) {
        const int h = i / kEndHalo, j = i % kEndHalo;
        const int hx = j % kEndHx, hy = (j / kEndHx) % kEndHy, hz = j / (kEndHx * kEndHy);
        const int xx = x0 - 1 + hx, yy = y0 - 1 + hy, zz = z - 1 + hz;
        uint4 v = make_uint4(0u, 0u, 0u, 0u);
        if (xx >= 0 && xx < X && yy >= 0 && yy < Y && zz >= 0 && zz < Z)
            v = *reinterpret_cast<const uint4*>(in + (((size_t)n * 2 + h) * plane + ((size_t)zz * Y + yy) * X + xx) * 8);
        halo[h][j] = v;
    }
    __syncthreads();
    const int tx = tid % kEndTx, ty = tid / kEndTx;
    const int x = x0 + tx, y = y0 + ty;
    if (x >= X || y >= Y) return;
    float acc = bias[0];
#pragma unroll 3
    for (int t = 0; t < 27; ++t) {
        const int j = ((t / 9) * kEndHy + ty + (t / 3) % 3) * kEndHx + tx + t % 3;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            float f[8];
            unpack_bf16x8(halo[h][j], f);
#pragma unroll
            for (int c = 0; c < 8; ++c) acc = fmaf(f[c], ws_[t * 16 + 8 * h + c], acc);
        }
    }
    const size_t i = (size_t)n * plane + ((size_t)z * Y + y) * X + x;
    out[i] = fmaf(scale, acc, vin[i]);
}

// Network input: chunk 0 of a 16-channel NC8 tensor = (v / scale, 0, ..., 0); chunk 1
// stays zero.  v: fp32 [n][z][y][x].
__global__ void prep_input_kernel(const float* __restrict__ v, float inv_scale, size_t plane, int batch,
                                  __nv_bfloat16* __restrict__ out) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)batch * plane) return;
    const size_t n = i / plane, p = i % plane;
    uint4 o;
    o.x = pack_bf16x2(v[i] * inv_scale, 0.f);
    o.y = o.z = o.w = 0u;
    *reinterpret_cast<uint4*>(out + ((n * 2) * plane + p) * 8) = o;
}

// 2x2x2 average of an NC8 tensor (X, Y, Z even) into the half-size grid.
__global__ void pool_kernel(const __nv_bfloat16* __restrict__ in, int X, int Y, int Z, int nchunks,
                            __nv_bfloat16* __restrict__ out) {
    const int x2 = X / 2, y2 = Y / 2, z2 = Z / 2;
    const size_t total = (size_t)nchunks * z2 * y2 * x2;
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    size_t t = i;
    const int x = t % x2;
    t /= x2;
    const int y = t % y2;
    t /= y2;
    const int z = t % z2;
    const size_t c = t / z2;
    float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int dz = 0; dz < 2; ++dz)
        for (int dy = 0; dy < 2; ++dy)
            for (int dx = 0; dx < 2; ++dx) {
                float f[8];
                unpack_bf16x8(*reinterpret_cast<const uint4*>(
                                  in + (((c * Z + 2 * z + dz) * Y + 2 * y + dy) * X + 2 * x + dx) * 8),
                              f);
#pragma unroll
                for (int j = 0; j < 8; ++j) s[j] += f[j];
            }
    uint4 o;
    o.x = pack_bf16x2(s[0] * 0.125f, s[1] * 0.125f);
    o.y = pack_bf16x2(s[2] * 0.125f, s[3] * 0.125f);
    o.z = pack_bf16x2(s[4] * 0.125f, s[5] * 0.125f);
    o.w = pack_bf16x2(s[6] * 0.125f, s[7] * 0.125f);
    *reinterpret_cast<uint4*>(out + i * 8) = o;
}

// Gradient through the average pool, plus the skip connection's gradient, times the
// ReLU mask of the pooled tensor: out[v] = (coarse[v / 2] / 8 + skip[v]) * (mask[v] > 0).
__global__ void pool_backward_kernel(const __nv_bfloat16* __restrict__ coarse, const __nv_bfloat16* __restrict__ skip,
                                     const __nv_bfloat16* __restrict__ mask, int X, int Y, int Z, int nchunks,
                                     __nv_bfloat16* __restrict__ out) {
    const size_t total = (size_t)nchunks * Z * Y * X;
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    size_t t = i;
    const int x = t % X;
    t /= X;
    const int y = t % Y;
    t /= Y;
    const int z = t % Z;
    const size_t c = t / Z;
    float g[8], s[8], m[8];
    unpack_bf16x8(*reinterpret_cast<const uint4*>(
                      coarse + (((c * (Z / 2) + z / 2) * (Y / 2) + y / 2) * (X / 2) + x / 2) * 8),
                  g);
    if (skip) unpack_bf16x8(*reinterpret_cast<const uint4*>(skip + i * 8), s);
    unpack_bf16x8(*reinterpret_cast<const uint4*>(mask + i * 8), m);
    float v[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        v[j] = g[j] * 0.125f + (skip ? s[j] : 0.f);
        v[j] = m[j] > 0.f ? v[j] : 0.f;
    }
    uint4 o;
    o.x = pack_bf16x2(v[0], v[1]);
    o.y = pack_bf16x2(v[2], v[3]);
    o.z = pack_bf16x2(v[4], v[5]);
    o.w = pack_bf16x2(v[6], v[7]);
    *reinterpret_cast<uint4*>(out + i * 8) = o;
}

// Nearest-neighbour upsampling by 2 of an NC8 tensor (coarse grid X/2, Y/2, Z/2).
// One thread per coarse cell: it reads the cell once and writes its 2 x 2 x 2 fine copies
// (X, Y, Z: the fine grid, even; the coarse grid has fewer than 2^32 cells).
__global__ void upsample_kernel(const __nv_bfloat16* __restrict__ in, int X, int Y, int Z, int nchunks,
                                __nv_bfloat16* __restrict__ out) {
    const uint32_t xc = (uint32_t)X / 2, yc = (uint32_t)Y / 2, zc = (uint32_t)Z / 2;
    const uint32_t total = (uint32_t)nchunks * zc * yc * xc;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    uint32_t t = i;
    const uint32_t x = t % xc;
    t /= xc;
    const uint32_t y = t % yc;
    t /= yc;
    const uint32_t z = t % zc;
    const uint32_t c = t / zc;
    const uint4 v = *reinterpret_cast<const uint4*>(in + (size_t)i * 8);
#pragma unroll
    for (int dz = 0; dz < 2; ++dz)
#pragma unroll
        for (int dy = 0; dy < 2; ++dy) {
            const size_t row = (((size_t)c * Z + 2 * z + dz) * Y + 2 * y + dy) * X + 2 * x;
            uint4* o = reinterpret_cast<uint4*>(out + row * 8);
            o[0] = v;
            o[1] = v;
        }
}

// Gradient through the upsampling (sum of the 8 children) times the ReLU mask of the
// coarse tensor.  X, Y, Z: coarse grid.
__global__ void upsample_backward_kernel(const __nv_bfloat16* __restrict__ fine, const __nv_bfloat16* __restrict__ mask,
                                         int X, int Y, int Z, int nchunks, __nv_bfloat16* __restrict__ out) {
    const size_t total = (size_t)nchunks * Z * Y * X;
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    size_t t = i;
    const int x = t % X;
    t /= X;
    const int y = t % Y;
    t /= Y;
    const int z = t % Z;
    const size_t c = t / Z;
    const int X2 = 2 * X, Y2 = 2 * Y, Z2 = 2 * Z;
    float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int dz = 0; dz < 2; ++dz)
        for (int dy = 0; dy < 2; ++dy)
            for (int dx = 0; dx < 2; ++dx) {
                float f[8];
                unpack_bf16x8(*reinterpret_cast<const uint4*>(
                                  fine + (((c * Z2 + 2 * z + dz) * Y2 + 2 * y + dy) * X2 + 2 * x + dx) * 8),
                              f);
#pragma unroll
                for (int j = 0; j < 8; ++j) s[j] += f[j];
            }
    float m[8];
    unpack_bf16x8(*reinterpret_cast<const uint4*>(mask + i * 8), m);
#pragma unroll
    for (int j = 0; j < 8; ++j) s[j] = m[j] > 0.f ? s[j] : 0.f;
    uint4 o;
    o.x = pack_bf16x2(s[0], s[1]);
    o.y = pack_bf16x2(s[2], s[3]);
    o.z = pack_bf16x2(s[4], s[5]);
    o.w = pack_bf16x2(s[6], s[7]);
    *reinterpret_cast<uint4*>(out + i * 8) = o;
}

// Loss gradient of L = mean(((out - target) / scale)^2) with respect to the normalised
// output y = out / scale, written as chunk 0 channel 0 of a 16-channel NC8 tensor (the
// head convolution's padded output); sum of squares to `loss` (FP64, one atomic per warp).
__global__ void loss_grad_kernel(const float* __restrict__ out, const float* __restrict__ target, float inv_scale,
                                 float grad_scale, size_t plane, int batch, __nv_bfloat16* __restrict__ dy,
                                 double* __restrict__ loss) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    double sq = 0.0;
    if (i < (size_t)batch * plane) {
        const float d = (out[i] - target[i]) * inv_scale;
        sq = (double)d * d;
        const size_t n = i / plane, p = i % plane;
        uint4 o;
        o.x = pack_bf16x2(grad_scale * d, 0.f);
        o.y = o.z = o.w = 0u;
        *reinterpret_cast<uint4*>(dy + ((n * 2) * plane + p) * 8) = o;
    }
    for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
    if ((threadIdx.x & 31) == 0 && sq != 0.0) atomicAdd(loss, sq);
}

// Adam on the FP32 master parameters.
__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, int n, float lr, float b1, float b2, float eps, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
}

// Kernel weight layouts from the FP32 master W[27][cout][cin_total]:
//  forward: [step][tap][half][N][8] with N = n_pad (>= cout), input channel
//           ci = step * 16 + half * 8 + j (zero beyond cin_total);
//  input gradient: [step][tap'][half][N'][8] for input channels ci0 .. ci0 + N' - 1,
//           output-gradient channel co = step * 16 + half * 8 + j (zero beyond cout),
//           W' = W[26 - tap'] transposed.
__global__ void relayout_forward_kernel(const float* __restrict__ W, int cout, int cin_total, int n_pad, int nsteps,
                                        __nv_bfloat16* __restrict__ out) {
    const int total = nsteps * 27 * 2 * n_pad * 8;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    int t = i;
    const int j = t % 8;
    t /= 8;
    const int nn = t % n_pad;
    t /= n_pad;
    const int half = t % 2;
    t /= 2;
    const int tap = t % 27;
    const int step = t / 27;
    const int ci = step * 16 + half * 8 + j;
    const float w = (nn < cout && ci < cin_total) ? W[((size_t)tap * cout + nn) * cin_total + ci] : 0.f;
    out[i] = __float2bfloat16_rn(w);
}
__global__ void relayout_backward_kernel(const float* __restrict__ W, int cout, int cin_total, int ci0, int n_part,
                                         int nsteps, __nv_bfloat16* __restrict__ out) {
    const int total = nsteps * 27 * 2 * n_part * 8;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    int t = i;
    const int j = t % 8;
    t /= 8;
    const int nn = t % n_part;
    t /= n_part;
    const int half = t % 2;
    t /= 2;
    const int tap = t % 27;
    const int step = t / 27;
    const int co = step * 16 + half * 8 + j;
    const int ci = ci0 + nn;
    const float w = co < cout ? W[((size_t)(26 - tap) * cout + co) * cin_total + ci] : 0.f;
    out[i] = __float2bfloat16_rn(w);
}

}  // namespace ws
