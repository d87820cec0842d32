// fg_common.cuh -- shared definitions for the femgpu sm_100a kernels.
//
// Layout of a DOF vector on the device ("native" layout): the lexicographic
// DOF grid (I fastest, then J, then K) of a structured hex mesh of order p,
// NI = nx*p+1, NJ = ny*p+1, NK = nz*p+1, with each I-row padded to a pitch
// NIp = round_up(NI, 4).  The pad entries are kept at zero.  The padding makes
// every row start 32-byte aligned, which the TMA tensor loads of the x tile
// require (global strides must be multiples of 16 bytes).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#define FG_MAXP 3

// device-side error bits (fg_op::d_err)
#define FG_DERR_TIMEOUT 1
#define FG_DERR_BOUNDS 2

namespace fg {

// 1-D basis tables at the Gauss points, index [p-1][q][d].
struct BasisTables {
    double B[FG_MAXP][FG_MAXP + 1][FG_MAXP + 1];
    double G[FG_MAXP][FG_MAXP + 1][FG_MAXP + 1];
    double gx[FG_MAXP][FG_MAXP + 1];  // Gauss points on [-1,1] for nq = p+1
    double gw[FG_MAXP][FG_MAXP + 1];  // Gauss weights
};

// Defined here: the library is a single translation unit.
__constant__ double c_B64[FG_MAXP][FG_MAXP + 1][FG_MAXP + 1];
__constant__ double c_G64[FG_MAXP][FG_MAXP + 1][FG_MAXP + 1];
__constant__ float c_B32[FG_MAXP][FG_MAXP + 1][FG_MAXP + 1];
__constant__ float c_G32[FG_MAXP][FG_MAXP + 1][FG_MAXP + 1];
// pairs for packed FP32 FMA (__ffma2_rn): (G, B), (B, G) and (B, B) per (p, q, d)
__constant__ float2 c_GB32[FG_MAXP][FG_MAXP + 1][FG_MAXP + 1];
__constant__ float2 c_BG32[FG_MAXP][FG_MAXP + 1][FG_MAXP + 1];
__constant__ float2 c_BB32[FG_MAXP][FG_MAXP + 1][FG_MAXP + 1];
// collocated derivative at the Gauss points, Dq = G B^-1: the derivative at
// point q of the degree-p polynomial through the values at the p+1 points
__constant__ float c_DQ32[FG_MAXP][FG_MAXP + 1][FG_MAXP + 1];
__constant__ double c_DQ64[FG_MAXP][FG_MAXP + 1][FG_MAXP + 1];

template <typename T> struct Tab;
template <> struct Tab<double> {
    static __device__ __forceinline__ double B(int p, int q, int d) { return c_B64[p - 1][q][d]; }
    static __device__ __forceinline__ double G(int p, int q, int d) { return c_G64[p - 1][q][d]; }
    static __device__ __forceinline__ double DQ(int p, int q, int k) { return c_DQ64[p - 1][q][k]; }
};
template <> struct Tab<float> {
    static __device__ __forceinline__ float B(int p, int q, int d) { return c_B32[p - 1][q][d]; }
    static __device__ __forceinline__ float G(int p, int q, int d) { return c_G32[p - 1][q][d]; }
    static __device__ __forceinline__ float DQ(int p, int q, int k) { return c_DQ32[p - 1][q][k]; }
};

__host__ __device__ constexpr int round_up(int a, int b) { return (a + b - 1) / b * b; }

// Geometry of the structured operator, shared by every kernel.
struct Grid {
    int nx, ny, nz, p;
    int NI, NJ, NK, NIp;   // DOF grid and padded row pitch
    int WY, TZ;            // tile: 32 elements in x (one warp), WY rows in y, TZ layers in z
    int ntx, nty, ntz;     // tiles per direction
    int ess;               // essential-face bits (tag t -> bit t-1: z0,z1,y0,y1,x0,x1)
    __host__ __device__ int64_t dof(int I, int J, int K) const {
        return ((int64_t)K * NJ + J) * NIp + I;
    }
    __host__ __device__ bool is_ess(int I, int J, int K) const {
        return ((ess & 1) && K == 0) || ((ess & 2) && K == NK - 1) ||
               ((ess & 4) && J == 0) || ((ess & 8) && J == NJ - 1) ||
               ((ess & 16) && I == 0) || ((ess & 32) && I == NI - 1);
    }
    __host__ __device__ int n_items() const { return ntx * nty * ntz; }
    // per-item face-slot sizes (x-hi, y-hi, z-hi planes of the item box)
    __host__ __device__ int fx() const { return (TZ * p + 1) * (WY * p + 1); }
    __host__ __device__ int fy() const { return (TZ * p + 1) * (32 * p + 1); }
    __host__ __device__ int fz() const { return (WY * p + 1) * (32 * p + 1); }
    __host__ __device__ int face_stride() const { return fx() + fy() + fz(); }
};

// ---------------------------------------------------------------------------
// PTX helpers: mbarrier, bulk async copies (TMA), timers.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}
__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
// Non-blocking test of a phase of an mbarrier.
__device__ __forceinline__ bool mbar_test_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, P1;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Potentially blocking test: the thread may be suspended until the phase
// completes or for at most about hint_ns nanoseconds.
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity, uint32_t hint_ns) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, P1;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(hint_ns)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}
// Wait for a phase of an mbarrier with a time limit.  On timeout the error
// word gets FG_DERR_TIMEOUT and false is returned; the caller stops issuing
// work and drains what it has in flight.  The first test does not block, and
// a suspended try never outlasts the limit, so a short limit is honoured.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int *err,
                                          uint64_t limit_ns = 1000000000ull) {
    if (mbar_test_wait(bar, parity)) return true;
    const uint32_t hint = (uint32_t)(limit_ns < 0xffffffffull ? limit_ns : 0xffffffffull);
    const uint64_t t0 = globaltimer_ns();
    while (true) {
        if (mbar_try_wait(bar, parity, hint)) return true;
        if (globaltimer_ns() - t0 > limit_ns) {
            if (err) atomicOr(err, FG_DERR_TIMEOUT);
            return false;
        }
    }
}
// Wait for stream stage `next - 1` of a producer's bulk copies while `ok`
// holds.  `waited` counts the stages whose data arrived; a stage whose wait ran
// out stays uncounted, so the drain after a timeout (drain_stages) still waits
// for the copy that was in flight.
__device__ __forceinline__ void wait_stage(uint64_t *bar, uint32_t parity, int *err, uint64_t limit_ns,
                                           bool &ok, int &waited, int next) {
    if (!ok) return;
    if (mbar_wait(bar, parity, err, limit_ns)) waited = next;
    else ok = false;
}
// After a timeout: wait (with the normal 1 s limit each) for every copy in
// [waited, issued) of a ring of `depth` mbarriers, so that no CTA exits while
// a bulk copy into its shared memory is still in flight.
__device__ __forceinline__ void drain_stages(uint64_t *bars, int depth, int waited, int issued) {
    for (int j = waited; j < issued; ++j) mbar_wait(&bars[j % depth], (j / depth) & 1, nullptr);
}
// Grid-wide barrier of a cooperative launch (every block resident at once),
// with a time limit.  bar[0] counts arrivals, bar[1] is the generation; the
// last block to arrive resets the count and advances the generation.  A block
// whose wait runs out sets FG_DERR_TIMEOUT, clears `ok` and from then on only
// arrives (never waits), so the launch ends within about one limit; the host
// then reports the timeout and clears bar[] before the next launch.
__device__ __forceinline__ void grid_barrier(unsigned *bar, int *err, bool &ok,
                                             uint64_t limit_ns = 1000000000ull) {
    __shared__ int ok_s;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok_s = ok ? 1 : 0;
        volatile unsigned *gen = bar + 1;
        const unsigned g = *gen;
        __threadfence();
        if (atomicAdd(bar, 1u) == gridDim.x - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else if (ok_s) {
            const uint64_t t0 = globaltimer_ns();
            while (*gen == g) {
                if (globaltimer_ns() - t0 > limit_ns) {
                    if (err) atomicOr(err, FG_DERR_TIMEOUT);
                    ok_s = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
    ok = ok_s != 0;
}
// 1-D bulk copy global -> shared, completing on an mbarrier (sizes/addresses
// must be multiples of 16 bytes).
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes,
                                         uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
// 3-D tiled tensor load global -> shared (no multicast).
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int c0, int c1,
                                            int c2, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], "
        "[%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void prefetch_tmap(const CUtensorMap *map) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

}  // namespace fg
