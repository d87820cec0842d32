// unet_tc.cuh -- the 3x3x3 convolution of the learned correction on the
// 5th-generation tensor cores: tcgen05.mma kind::f16 with BF16 operands in
// shared memory and FP32 accumulators in tensor memory (TMEM).
//
// Implicit GEMM  out[v][n] = bias[n] + sum_{tap, ci} W[n][tap*Cin + ci] * in[v + off(tap)][ci]
// (the same product as conv3_fwd_kernel, 0 outside the volume).  One CTA of
// 128 threads owns 128 voxels (M = 128: voxel m of the tile is TMEM lane m)
// and every output channel (N = cout rounded up to 16: TMEM columns).  The K
// loop runs over the 27 taps.  For each tap the 128 threads stage the operands
// in shared memory -- thread m copies voxel m's neighbour channels with
// 16-byte cp.async (zero-filled outside the volume and in the padding
// channels), and the tap's weight rows W[n][tap*Cin .. tap*Cin + Cin) are
// copied alongside -- then one thread issues the taps' CinP/16 MMAs each
// (K = 16) and commits them to the stage's mbarrier.  A stage holds G = 1, 3
// or 9 taps, and the stages form a ring of S = 2..8: the copies of a tap group
// are issued S - 2 groups ahead, so the gathers of several taps are in flight
// while the tensor core works, and a stage is refilled only after the commit
// of the MMAs that read it has arrived.  The epilogue reads the accumulators with tcgen05.ld (warp w owns
// lanes 32w .. 32w+31, i.e. its threads' voxels), adds the bias, applies ReLU
// and stores BF16.
//
// Canonical K-major operand layout without swizzle, [R rows][CinP] BF16: core
// matrices of 8 rows x 16 bytes (8 values), element (r, k) at byte
//   (r / 8) * SBO + (k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2,   SBO = CinP * 16,
// so the K-slice [16 j, 16 j + 16) is described by start byte 256 j, leading
// byte offset 128 (the second 8-value half of the slice) and stride byte
// offset SBO (the next 8 rows).
//
// Every mbarrier wait is bounded (mbar_wait): on timeout the error word gets
// FG_DERR_TIMEOUT, the CTA stops issuing, waits (bounded) for the commits it
// has in flight, frees its TMEM and returns without storing.
#pragma once
#include <cuda_bf16.h>

#include "unet_kernels.cuh"

namespace fg {

// Shared-memory matrix descriptor: start address, leading byte offset 128,
// stride byte offset `sbo` (all in 16-byte units), descriptor version 1,
// base offset 0, no swizzle.
__device__ __forceinline__ uint64_t umma_desc_kmajor(uint32_t saddr, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128u >> 4) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator (bits 4-5 = 1), A and
// B BF16 (bits 7-9, 10-12 = 1), both K-major (bits 15, 16 = 0), N >> 3 in bits
// 17-22, M >> 4 in bits 24-28.
template <int N>
__host__ __device__ constexpr uint32_t umma_idesc_bf16_m128() {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}
// The mbarrier receives one arrival once every MMA this thread issued before
// has completed (its shared-memory operands are then free to overwrite).
__device__ __forceinline__ void umma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after_sync() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// Whole-warp TMEM allocation of `ncols` columns (a power of two >= 32); the
// base address is written to shared memory.
__device__ __forceinline__ void tmem_alloc_warp(uint32_t *dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc_warp(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
// 32 lanes x 16 consecutive 32-bit columns: thread t of the warp gets lane
// (lane field of taddr) + t, register j = column (column field of taddr) + j.
__device__ __forceinline__ void tmem_ld_32x32b_x16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
        "%13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

constexpr int TC_MAX_CINP = 112;  // largest padded input channel count (C2 + C1 <= 112)
constexpr int TC_MAX_STAGES = 8;

// TMEM columns a CTA allocates for N accumulator columns.
__host__ __device__ constexpr uint32_t tc_tmem_cols(int npad) { return npad <= 32 ? 32u : (npad <= 64 ? 64u : 128u); }

// 16-byte asynchronous copy global -> shared; src_bytes = 0 writes zeros
// (the source address must still be a valid one).
__device__ __forceinline__ void cp_async16(void *dst, const void *src, uint32_t src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// Wait until at most n of this thread's most recent copy groups are pending.
__device__ __forceinline__ void cp_async_wait(int n) {
    switch (n) {  // the operand is an immediate
    case 0: asm volatile("cp.async.wait_group 0;" ::: "memory"); break;
    case 1: asm volatile("cp.async.wait_group 1;" ::: "memory"); break;
    case 2: asm volatile("cp.async.wait_group 2;" ::: "memory"); break;
    case 3: asm volatile("cp.async.wait_group 3;" ::: "memory"); break;
    case 4: asm volatile("cp.async.wait_group 4;" ::: "memory"); break;
    case 5: asm volatile("cp.async.wait_group 5;" ::: "memory"); break;
    default: asm volatile("cp.async.wait_group 6;" ::: "memory"); break;
    }
}

// Requirements (checked by the host): Cin, cout multiples of 8; CinP = Cin
// rounded up to 16 (<= TC_MAX_CINP); NPAD = cout rounded up to 16; channel
// strides and offsets of both views multiples of 8 (16-byte accesses); Kp a
// multiple of 16 (weight rows 32-byte aligned); G in {1, 3, 9} taps per
// stage; 2 <= S <= TC_MAX_STAGES stages.  Dynamic shared memory holds S
// stages of G taps, each tap (128 + NPAD) x CinP BF16 values.
//
// Schedule: the 27 taps form NG = 27 / G groups; group g lives in stage
// g % S.  Its copies are issued D = S - 2 groups ahead (one cp.async group per
// tap group), into a stage whose previous group's MMAs were committed at least
// two iterations earlier, so the refill rarely waits on the tensor core; one
// barrier per group, so a conv of small volumes (a few CTAs) pays NG rounds of
// gather latency instead of 27.
template <int NPAD>
__global__ void __launch_bounds__(128) conv3_fwd_tc_kernel(const TView in, const Vol V, int Cin, int CinP,
                                                           const __nv_bfloat16 *__restrict__ W, int Kp,
                                                           int cout, const float *__restrict__ bias,
                                                           TView out, int relu, int G, int S, int *err) {
    constexpr uint32_t NCOLS = tc_tmem_cols(NPAD);
    constexpr uint32_t IDESC = umma_idesc_bf16_m128<NPAD>();
    extern __shared__ __align__(1024) unsigned char tc_smem[];
    __shared__ uint64_t bars[TC_MAX_STAGES];
    __shared__ uint32_t tmem_base_s;
    const int tid = threadIdx.x, warp = tid >> 5;
    const uint32_t sbo = (uint32_t)CinP * 16u;
    const uint32_t a_bytes = 128u * sbo / 8u, tap_bytes = a_bytes + (uint32_t)NPAD * sbo / 8u;
    const uint32_t stage_bytes = tap_bytes * (uint32_t)G;
    const int nc8 = CinP / 8, c8in = Cin / 8, nk16 = CinP / 16;
    const int NG = 27 / G, D = S - 2;

    if (warp == 0) tmem_alloc_warp(&tmem_base_s, NCOLS);
    if (tid == 0) {
        for (int s = 0; s < S; ++s) mbar_init(&bars[s], 1);
        fence_barrier_init();
    }
    tc_fence_before_sync();
    __syncthreads();
    tc_fence_after_sync();
    const uint32_t tmem = tmem_base_s;

    const int64_t nv = V.nvox();
    const int64_t v = (int64_t)blockIdx.x * 128 + tid;
    const bool vok = v < nv;
    int b, z, y, x;
    vox_coords(V, vok ? v : 0, b, z, y, x);
    const __nv_bfloat16 *vbase = in.p + in.co;  // a valid source for zero-filled copies

    // copies of tap group gi into its stage: per tap, this thread's voxel row
    // and the weight rows (n fastest)
    auto issue_group = [&](int gi) {
        unsigned char *st = tc_smem + (gi % S) * stage_bytes;
        for (int j = 0; j < G; ++j) {
            const int u = gi * G + j;
            unsigned char *As = st + j * tap_bytes, *Bs = As + a_bytes;
            const int dz = u / 9 - 1, dy = (u / 3) % 3 - 1, dx = u % 3 - 1;
            const int zz = z + dz, yy = y + dy, xx = x + dx;
            const bool inb = vok && zz >= 0 && zz < V.Z && yy >= 0 && yy < V.Y && xx >= 0 && xx < V.X;
            const __nv_bfloat16 *src =
                inb ? in.p + ((((int64_t)b * V.Z + zz) * V.Y + yy) * V.X + xx) * in.cs + in.co : vbase;
            unsigned char *arow = As + (tid >> 3) * sbo + (tid & 7) * 16;
            for (int c8 = 0; c8 < nc8; ++c8) {
                const bool live = inb && c8 < c8in;
                cp_async16(arow + c8 * 128, live ? src + c8 * 8 : vbase, live ? 16u : 0u);
            }
            for (int i = tid; i < NPAD * nc8; i += 128) {
                const int c8 = i / NPAD, n = i - c8 * NPAD;
                const bool live = n < cout && c8 < c8in;
                cp_async16(Bs + (n >> 3) * sbo + c8 * 128 + (n & 7) * 16,
                           live ? W + (int64_t)n * Kp + u * Cin + c8 * 8 : W, live ? 16u : 0u);
            }
        }
    };

    bool ok = true;
    for (int gi = 0; gi < D && gi < NG; ++gi) {
        issue_group(gi);
        cp_async_commit();
    }
    int issued = 0;  // tap groups whose MMAs have been committed
    for (int t = 0; t < NG; ++t) {
        const int gu = t + D;
        if (gu < NG) {
            // stage gu % S last held group gu - S, whose MMAs were committed at iteration gu - S <= t - 2
            if (gu >= S) ok = mbar_wait(&bars[gu % S], ((gu - S) / S) & 1, err) && ok;
            issue_group(gu);
        }
        cp_async_commit();  // one group per iteration (empty past the last): group t's copies are complete
        cp_async_wait(D);   // once at most D newer groups are pending
        fence_proxy_async();  // async-proxy reads of the staged operands follow
        ok = __syncthreads_and(ok) != 0;
        if (!ok) break;
        if (tid == 0) {
            tc_fence_after_sync();
            const uint32_t s0 = smem_u32(tc_smem + (t % S) * stage_bytes);
            for (int j = 0; j < G; ++j) {
                const uint32_t a0 = s0 + j * tap_bytes, b0 = a0 + a_bytes;
                for (int k = 0; k < nk16; ++k)
                    umma_bf16(tmem, umma_desc_kmajor(a0 + 256u * k, sbo), umma_desc_kmajor(b0 + 256u * k, sbo),
                              IDESC, (t | j | k) != 0);
            }
            umma_commit(&bars[t % S]);
        }
        issued = t + 1;
    }
    cp_async_wait(0);  // no copy into shared memory outlives the CTA
    // the last commit of every stage has not been waited for (waiting again on
    // a completed last phase returns at once)
    bool done = true;
    for (int s = 0; s < S && s < issued; ++s) {
        const int last = s + S * ((issued - 1 - s) / S);
        done = mbar_wait(&bars[s], (last / S) & 1, err) && done;
    }
    ok = __syncthreads_and(ok && done && issued == NG) != 0;
    tc_fence_after_sync();
    if (ok) {
        const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
#pragma unroll
        for (int c = 0; c < NPAD / 16; ++c) {
            uint32_t r[16];
            tmem_ld_32x32b_x16(tmem + lane_base + (uint32_t)(c * 16), r);
            if (vok) {
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int n0 = 16 * c + 8 * h;
                    if (n0 < cout) {
                        uint32_t pk[4];
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            float f0 = __uint_as_float(r[8 * h + 2 * q]), f1 = __uint_as_float(r[8 * h + 2 * q + 1]);
                            if (bias) {
                                f0 += bias[n0 + 2 * q];
                                f1 += bias[n0 + 2 * q + 1];
                            }
                            if (relu) {
                                f0 = fmaxf(f0, 0.f);
                                f1 = fmaxf(f1, 0.f);
                            }
                            const __nv_bfloat162 p2 = __floats2bfloat162_rn(f0, f1);
                            pk[q] = *reinterpret_cast<const uint32_t *>(&p2);
                        }
                        *reinterpret_cast<uint4 *>(out.p + v * out.cs + out.co + n0) =
                            make_uint4(pk[0], pk[1], pk[2], pk[3]);
                    }
                }
            }
        }
    }
    tc_fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after_sync();
        tmem_dealloc_warp(tmem, NCOLS);
    }
}

// Taps per stage and stages of one launch: the largest G in {9, 3, 1} for
// which two stages fit the budget (about 200 KB -- one CTA per SM -- when the
// grid has at most one CTA per SM, else about 110 KB, two per SM), then as
// many stages as the budget holds (2 to 8, at most one more than the groups).
static inline void conv_tc_plan(int npad, int cinp, int64_t blocks, int &G, int &S) {
    const size_t tap = (size_t)(128 + npad) * cinp * 2;
    const size_t budget = blocks <= 148 ? 200 * 1024 : 110 * 1024;
    G = 1;
    if (2 * 9 * tap <= budget) G = 9;
    else if (2 * 3 * tap <= budget) G = 3;
    const int NG = 27 / G;
    size_t s = budget / (G * tap);
    if (s < 2) s = 2;
    if (s > (size_t)TC_MAX_STAGES) s = TC_MAX_STAGES;
    if (s > (size_t)NG + 1) s = NG + 1;
    S = (int)s;
}
// Dynamic shared memory of one CTA, raised where needed so that no more CTAs
// fit on an SM than their TMEM allocations (512 columns per SM) allow -- an
// allocation never has to wait for another CTA to free columns.
static inline size_t conv_tc_smem_bytes(int npad, int cinp, int G, int S) {
    size_t need = (size_t)S * G * (128 + npad) * cinp * 2;
    const int maxc = 512 / (int)tc_tmem_cols(npad);
    if (maxc < 16) {  // 16 CTAs of 128 threads already fill an SM's 2048 threads
        const size_t cap = 233472 / (size_t)(maxc + 1) - 1024 + 16;
        if (need < cap) need = cap;
    }
    return need;
}
constexpr size_t TC_SMEM_MAX = 220 * 1024;  // above every request (the budgets plus one stage of rounding)

}  // namespace fg
