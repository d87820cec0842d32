// vec_kernels.cuh -- fused vector updates of the PCG / Chebyshev / power
// iterations on native-layout DOF vectors.
//
// Every reduction is deterministic: a fixed grid (VEC_GRID blocks, independent
// of timing) writes one partial per block; the block that finishes last (an
// atomic ticket) sums the partials in index order and updates the solver
// scalars on the device.  No host round trip per iteration: the host only
// polls `done` every few iterations, and every kernel returns at once once
// `done` is set, so the iteration count equals that of a per-iteration check
// (crates/parallel/src/par_solver.rs:310-322).
#pragma once
#include "fg_common.cuh"

namespace fg {

constexpr int VEC_THREADS = 256;
constexpr int VEC_GRID = 592;  // fixed: the reduction order must not depend on the device

struct SolverState {
    double rz, pap, alpha, beta, rr, bb, bnorm, res;
    double rtol, atol;
    double rho;                // power iteration: ||w||
    double tmp[4];
    double maxr, delta;        // reliable updates: residual norm at the last update, trigger ratio
    int iter, done, converged, breakdown, max_iter;
    int trigger, skip_rel;     // reliable update pending / its kernels skip
    unsigned int ticket;
    // operator-CG stopping rule (solve_cg_operator, crates/solver/src/lib.rs:229-278):
    // converged when ||r|| <= stop_abs = max(atol, rtol*max(||b||, 1e-32)), also
    // before the first iteration; breakdown |pAp| < 1e-32; res = ||r|| (absolute)
    int cgop;
    double stop_abs;
};

template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double *sm) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int NW = VEC_THREADS / 32;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double s = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) sm[k * NW + warp] = s;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double s = lane < NW ? sm[k * NW + lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            v[k] = s;
        }
    }
    __syncthreads();
}

// Writes this block's partials; returns true in the last block, whose thread 0
// then holds the grand totals in `tot` (summed in block order).
template <int NV>
__device__ __forceinline__ bool grid_sum(double (&v)[NV], double *partials, SolverState *st,
                                         double (&tot)[NV]) {
    __shared__ double sm[NV * (VEC_THREADS / 32)];
    __shared__ int last;
    block_sum<NV>(v, sm);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) partials[blockIdx.x * NV + k] = v[k];
        __threadfence();
        const unsigned t = atomicAdd(&st->ticket, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    double acc[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) acc[k] = 0.0;
    // fixed order: thread i sums blocks i, i+256, ... then a fixed tree
    for (int b = threadIdx.x; b < (int)gridDim.x; b += VEC_THREADS)
#pragma unroll
        for (int k = 0; k < NV; ++k) acc[k] += __ldcg(&partials[b * NV + k]);
    block_sum<NV>(acc, sm);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) tot[k] = acc[k];
        st->ticket = 0;
    }
    return true;
}

#define FG_VEC_LOOP(i, n) \
    for (int64_t i = (int64_t)blockIdx.x * VEC_THREADS + threadIdx.x; i < (n); i += (int64_t)gridDim.x * VEC_THREADS)

// 4-wide groups: native vectors have a length that is a multiple of 4 (the row
// pitch is), and cudaMalloc alignment makes every group 16/32-byte aligned.
template <typename T> struct alignas(4 * sizeof(T)) V4 { T a[4]; };
template <typename T> __device__ __forceinline__ V4<T> ld4(const T *p, int64_t q) {
    return reinterpret_cast<const V4<T> *>(p)[q];
}
template <typename T> __device__ __forceinline__ void st4(T *p, int64_t q, const V4<T> &v) {
    reinterpret_cast<V4<T> *>(p)[q] = v;
}
#define FG_VEC4_LOOP(q, n)                                                                  \
    for (int64_t q = (int64_t)blockIdx.x * VEC_THREADS + threadIdx.x; q < ((n) >> 2);       \
         q += (int64_t)gridDim.x * VEC_THREADS)
#define FG_K4 _Pragma("unroll") for (int k = 0; k < 4; ++k)

// r = b - ap; z = dinv r (jacobi) ; p = z ; rz = r.z ; bb = b.b
template <typename T>
__global__ void __launch_bounds__(VEC_THREADS) k_pcg_init(int64_t n, const T *__restrict__ b,
                                                          const T *__restrict__ ap,
                                                          const T *__restrict__ dinv,
                                                          T *__restrict__ r, T *__restrict__ z,
                                                          T *__restrict__ p, int jacobi,
                                                          double *partials, SolverState *st) {
    double v[2] = {0.0, 0.0};
    FG_VEC4_LOOP(q, n) {
        const V4<T> bv = ld4(b, q), av = ld4(ap, q);
        V4<T> rv, zv, dv;
        if (jacobi) dv = ld4(dinv, q);
        FG_K4 {
            rv.a[k] = bv.a[k] - av.a[k];
            v[1] += (double)bv.a[k] * (double)bv.a[k];
            if (jacobi) {
                zv.a[k] = dv.a[k] * rv.a[k];
                v[0] += (double)rv.a[k] * (double)zv.a[k];
            }
        }
        st4(r, q, rv);
        if (jacobi) {
            st4(z, q, zv);
            st4(p, q, zv);
        }
    }
    double tot[2];
    if (grid_sum<2>(v, partials, st, tot) && threadIdx.x == 0) {
        st->rz = tot[0];
        st->bb = tot[1];
        st->bnorm = sqrt(tot[1]);
        st->iter = 0;
        st->converged = 0;
        st->breakdown = 0;
        st->done = 0;
        if (st->cgop) {  // z = r here, so rz = ||r0||^2
            st->stop_abs = fmax(st->atol, st->rtol * fmax(st->bnorm, 1e-32));
            st->res = sqrt(tot[0]);
            if (st->res <= st->stop_abs) {
                st->converged = 1;
                st->done = 1;
            }
        } else if (st->bnorm < 1e-30) {
            st->converged = 1;
            st->done = 1;
            st->res = 0.0;
        }
    }
}

// pap = p.ap ; alpha = rz / pap  (breakdown if |pap| < 1e-30)
template <typename T>
__global__ void __launch_bounds__(VEC_THREADS) k_pcg_pap(int64_t n, const T *__restrict__ p,
                                                         const T *__restrict__ ap,
                                                         double *partials, SolverState *st) {
    if (st->done) return;
    double v[1] = {0.0};
    FG_VEC4_LOOP(q, n) {
        const V4<T> pv = ld4(p, q), av = ld4(ap, q);
        FG_K4 v[0] += (double)pv.a[k] * (double)av.a[k];
    }
    double tot[1];
    if (grid_sum<1>(v, partials, st, tot) && threadIdx.x == 0) {
        st->pap = tot[0];
        if (fabs(tot[0]) < (st->cgop ? 1e-32 : 1e-30)) {
            st->breakdown = 1;
            st->done = 1;
        } else {
            st->alpha = st->rz / tot[0];
        }
    }
}

// x += alpha p ; r -= alpha ap ; [jacobi: z = dinv r, rz_new] ; rr ; convergence
template <typename T>
__global__ void __launch_bounds__(VEC_THREADS) k_pcg_update(int64_t n, T *__restrict__ x,
                                                            T *__restrict__ r,
                                                            const T *__restrict__ p,
                                                            const T *__restrict__ ap,
                                                            const T *__restrict__ dinv,
                                                            T *__restrict__ z, int jacobi,
                                                            double *partials, SolverState *st) {
    if (st->done) return;
    const T alpha = (T)st->alpha;
    double v[2] = {0.0, 0.0};
    FG_VEC4_LOOP(q, n) {
        V4<T> xv = ld4(x, q), rv = ld4(r, q);
        const V4<T> pv = ld4(p, q), av = ld4(ap, q);
        V4<T> dv, zv;
        if (jacobi) dv = ld4(dinv, q);
        FG_K4 {
            xv.a[k] += alpha * pv.a[k];
            rv.a[k] = rv.a[k] - alpha * av.a[k];
            v[0] += (double)rv.a[k] * (double)rv.a[k];
            if (jacobi) {
                zv.a[k] = dv.a[k] * rv.a[k];
                v[1] += (double)rv.a[k] * (double)zv.a[k];
            }
        }
        st4(x, q, xv);
        st4(r, q, rv);
        if (jacobi) st4(z, q, zv);
    }
    double tot[2];
    if (grid_sum<2>(v, partials, st, tot) && threadIdx.x == 0) {
        st->iter += 1;
        st->rr = tot[0];
        const double rn = sqrt(tot[0]);
        st->res = st->cgop ? rn : rn / st->bnorm;
        if (st->cgop ? rn <= st->stop_abs : (st->res < st->rtol || rn < st->atol)) {
            st->converged = 1;
            st->done = 1;
        } else if (st->iter >= st->max_iter) {
            st->done = 1;
        } else if (jacobi) {
            st->beta = tot[1] / st->rz;
            st->rz = tot[1];
        }
    }
}

// ---- one PCG iteration's vector work in one cooperative launch -----------
// The block partials of a reduction, then a grid barrier, then every block
// sums all partials in the order grid_sum's last block uses, so every block
// holds the same totals, bit for bit those of the separate kernels.
template <int NV>
__device__ __forceinline__ void all_blocks_sum(double (&v)[NV], double *partials, unsigned *bar, int *err,
                                               bool &ok, double (&tot)[NV]) {
    __shared__ double sm[NV * (VEC_THREADS / 32)];
    __shared__ double tb[NV];
    block_sum<NV>(v, sm);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) partials[blockIdx.x * NV + k] = v[k];
    }
    grid_barrier(bar, err, ok);
    double acc[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) acc[k] = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += VEC_THREADS)
#pragma unroll
        for (int k = 0; k < NV; ++k) acc[k] += __ldcg(&partials[b * NV + k]);
    block_sum<NV>(acc, sm);
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) tb[k] = acc[k];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; ++k) tot[k] = tb[k];
}

// k_pcg_pap + k_pcg_update (Jacobi: z = dinv r) + k_pcg_pupdate of one
// iteration in one launch with two grid barriers: p.Ap and alpha, the x / r /
// z update with r.r and r.z, the stopping test, beta and p = z + beta p --
// the iteration of par_solve_pcg_jacobi (crates/parallel/src/par_solver.rs:
// 296-330) and of solve_cg_operator (dinv = 1, its own stopping rule).  The
// state is read by every block at entry and written by block 0 only; the two
// reductions use separate partial regions.  Same values as the separate kernels.
template <typename T>
__global__ void __launch_bounds__(VEC_THREADS) k_pcg_fused_jacobi(int64_t n, T *__restrict__ x, T *__restrict__ r,
                                                                  T *__restrict__ p, const T *__restrict__ ap,
                                                                  const T *__restrict__ dinv, T *__restrict__ z,
                                                                  double *partials, SolverState *st, unsigned *bar,
                                                                  int *err) {
    if (st->done) return;
    const double rz0 = st->rz, bnorm = st->bnorm, rtol = st->rtol, atol = st->atol, stop_abs = st->stop_abs;
    const int iter0 = st->iter, max_iter = st->max_iter, cgop = st->cgop;
    bool ok = true;
    double v1[1] = {0.0};
    FG_VEC4_LOOP(q, n) {
        const V4<T> pv = ld4(p, q), av = ld4(ap, q);
        FG_K4 v1[0] += (double)pv.a[k] * (double)av.a[k];
    }
    double pap[1];
    all_blocks_sum<1>(v1, partials, bar, err, ok, pap);
    if (fabs(pap[0]) < (cgop ? 1e-32 : 1e-30)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            st->pap = pap[0];
            st->breakdown = 1;
            st->done = 1;
        }
        return;
    }
    const double alpha_d = rz0 / pap[0];
    const T alpha = (T)alpha_d;
    double v2[2] = {0.0, 0.0};
    FG_VEC4_LOOP(q, n) {
        V4<T> xv = ld4(x, q), rv = ld4(r, q), zv;
        const V4<T> pv = ld4(p, q), av = ld4(ap, q), dv = ld4(dinv, q);
        FG_K4 {
            xv.a[k] += alpha * pv.a[k];
            rv.a[k] = rv.a[k] - alpha * av.a[k];
            v2[0] += (double)rv.a[k] * (double)rv.a[k];
            zv.a[k] = dv.a[k] * rv.a[k];
            v2[1] += (double)rv.a[k] * (double)zv.a[k];
        }
        st4(x, q, xv);
        st4(r, q, rv);
        st4(z, q, zv);
    }
    double tot[2];
    all_blocks_sum<2>(v2, partials + 2 * VEC_GRID, bar, err, ok, tot);
    const double rn = sqrt(tot[0]);
    const double res = cgop ? rn : rn / bnorm;
    const bool converged = cgop ? rn <= stop_abs : (res < rtol || rn < atol);
    const bool stop = converged || iter0 + 1 >= max_iter;
    const double beta_d = tot[1] / rz0;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        st->pap = pap[0];
        st->alpha = alpha_d;
        st->iter = iter0 + 1;
        st->rr = tot[0];
        st->res = res;
        if (converged) {
            st->converged = 1;
            st->done = 1;
        } else if (stop) {
            st->done = 1;
        } else {
            st->beta = beta_d;
            st->rz = tot[1];
        }
    }
    if (stop) return;
    const T beta = (T)beta_d;
    FG_VEC4_LOOP(q, n) {
        const V4<T> zv = ld4(z, q);
        V4<T> pv = ld4(p, q);
        FG_K4 pv.a[k] = zv.a[k] + beta * pv.a[k];
        st4(p, q, pv);
    }
}

// rz_new = r.z ; beta = rz_new / rz ; rz = rz_new   (non-Jacobi preconditioners)
template <typename T>
__global__ void __launch_bounds__(VEC_THREADS) k_pcg_rz(int64_t n, const T *__restrict__ r,
                                                        const T *__restrict__ z,
                                                        double *partials, SolverState *st, int init) {
    if (st->done) return;
    double v[1] = {0.0};
    FG_VEC4_LOOP(q, n) {
        const V4<T> rv = ld4(r, q), zv = ld4(z, q);
        FG_K4 v[0] += (double)rv.a[k] * (double)zv.a[k];
    }
    double tot[1];
    if (grid_sum<1>(v, partials, st, tot) && threadIdx.x == 0) {
        if (!init) st->beta = tot[0] / st->rz;
        st->rz = tot[0];
    }
}

// p = z + beta p   (init: p = z)
template <typename T>
__global__ void __launch_bounds__(VEC_THREADS) k_pcg_pupdate(int64_t n, const T *__restrict__ z,
                                                             T *__restrict__ p,
                                                             const SolverState *st, int init) {
    if (st->done) return;
    const T beta = init ? T(0) : (T)st->beta;
    FG_VEC4_LOOP(q, n) {
        const V4<T> zv = ld4(z, q);
        // the first direction is z itself: the previous contents of p (a
        // finished solve's, possibly not finite) are not read
        V4<T> pv = init ? zv : ld4(p, q);
        if (!init) {
            FG_K4 pv.a[k] = zv.a[k] + beta * pv.a[k];
        }
        st4(p, q, pv);
    }
}

// Chebyshev sweep 1 from zero: res = dinv r ; d = res / theta ; z = d
template <typename T>
__global__ void __launch_bounds__(VEC_THREADS) k_cheb_first(int64_t n, const T *__restrict__ r,
                                                            const T *__restrict__ dinv,
                                                            T *__restrict__ res,
                                                            T *__restrict__ d,
                                                            T *__restrict__ z, double inv_theta,
                                                            const SolverState *st) {
    if (st && st->done) return;
    const T it = (T)inv_theta;
    FG_VEC4_LOOP(q, n) {
        const V4<T> rv = ld4(r, q), dv = ld4(dinv, q);
        V4<T> sv, dd;
        FG_K4 {
            sv.a[k] = dv.a[k] * rv.a[k];
            dd.a[k] = sv.a[k] * it;
        }
        st4(res, q, sv);
        st4(d, q, dd);
        st4(z, q, dd);
    }
}

// Chebyshev sweep: res -= dinv t ; d = c1 d + c2 res ; z += d
template <typename T>
__global__ void __launch_bounds__(VEC_THREADS) k_cheb_step(int64_t n, const T *__restrict__ t,
                                                           const T *__restrict__ dinv,
                                                           T *__restrict__ res,
                                                           T *__restrict__ d,
                                                           T *__restrict__ z, double c1,
                                                           double c2, const SolverState *st) {
    if (st && st->done) return;
    const T a1 = (T)c1, a2 = (T)c2;
    FG_VEC4_LOOP(q, n) {
        const V4<T> tv = ld4(t, q), dv = ld4(dinv, q);
        V4<T> sv = ld4(res, q), dd = ld4(d, q), zv = ld4(z, q);
        FG_K4 {
            sv.a[k] = sv.a[k] - dv.a[k] * tv.a[k];
            dd.a[k] = a1 * dd.a[k] + a2 * sv.a[k];
            zv.a[k] += dd.a[k];
        }
        st4(res, q, sv);
        st4(d, q, dd);
        st4(z, q, zv);
    }
}

// The same sweeps with each d_k kept in its own vector and z formed once, in
// the last sweep: z = d_0 + d_1 + ... + d_s added in that order, the order in
// which k_cheb_step accumulates it, so z is bit-identical.  Per application of
// degree s + 1 this moves 6 s + 5 vector passes instead of 8 s + 5 -- the last
// sweep writes neither res nor d, and z is written once instead of s + 1 times.
constexpr int CHEB_MAXD = 16;  // longest list of earlier d_k the last sweep sums
template <typename T> struct ChebSum {
    const T *d[CHEB_MAXD];  // d_0 .. d_{s-2}
    int n;
};

// sweep 1 from zero: res = dinv r ; d_0 = res / theta
template <typename T>
__global__ void __launch_bounds__(VEC_THREADS) k_cheb_first_d(int64_t n, const T *__restrict__ r,
                                                              const T *__restrict__ dinv,
                                                              T *__restrict__ res, T *__restrict__ d,
                                                              double inv_theta, const SolverState *st) {
    if (st && st->done) return;
    const T it = (T)inv_theta;
    FG_VEC4_LOOP(q, n) {
        const V4<T> rv = ld4(r, q), dv = ld4(dinv, q);
        V4<T> sv, dd;
        FG_K4 {
            sv.a[k] = dv.a[k] * rv.a[k];
            dd.a[k] = sv.a[k] * it;
        }
        st4(res, q, sv);
        st4(d, q, dd);
    }
}

// middle sweep: res -= dinv t ; d_k = c1 d_{k-1} + c2 res
template <typename T>
__global__ void __launch_bounds__(VEC_THREADS) k_cheb_mid(int64_t n, const T *__restrict__ t,
                                                          const T *__restrict__ dinv,
                                                          T *__restrict__ res,
                                                          const T *__restrict__ dprev,
                                                          T *__restrict__ dnext, double c1, double c2,
                                                          const SolverState *st) {
    if (st && st->done) return;
    const T a1 = (T)c1, a2 = (T)c2;
    FG_VEC4_LOOP(q, n) {
        const V4<T> tv = ld4(t, q), dv = ld4(dinv, q), pv = ld4(dprev, q);
        V4<T> sv = ld4(res, q), dd;
        FG_K4 {
            sv.a[k] = sv.a[k] - dv.a[k] * tv.a[k];
            dd.a[k] = a1 * pv.a[k] + a2 * sv.a[k];
        }
        st4(res, q, sv);
        st4(dnext, q, dd);
    }
}

// last sweep: d_s = c1 d_{s-1} + c2 (res - dinv t) ; z = d_0 + ... + d_{s-1} + d_s
template <typename T>
__global__ void __launch_bounds__(VEC_THREADS) k_cheb_last(int64_t n, const T *__restrict__ t,
                                                           const T *__restrict__ dinv,
                                                           const T *__restrict__ res,
                                                           const T *__restrict__ dprev,
                                                           const ChebSum<T> earlier, T *__restrict__ z,
                                                           double c1, double c2, const SolverState *st) {
    if (st && st->done) return;
    const T a1 = (T)c1, a2 = (T)c2;
    FG_VEC4_LOOP(q, n) {
        const V4<T> tv = ld4(t, q), dv = ld4(dinv, q), pv = ld4(dprev, q), sv = ld4(res, q);
        V4<T> zv = earlier.n > 0 ? ld4(earlier.d[0], q) : pv;
        for (int j = 1; j < earlier.n; ++j) {
            const V4<T> w = ld4(earlier.d[j], q);
            FG_K4 zv.a[k] += w.a[k];
        }
        FG_K4 {
            if (earlier.n > 0) zv.a[k] += pv.a[k];
            const T rs = sv.a[k] - dv.a[k] * tv.a[k];
            const T dk = a1 * pv.a[k] + a2 * rs;
            zv.a[k] += dk;
        }
        st4(z, q, zv);
    }
}

// ||b - ap|| / bnorm into st->tmp[0] (true residual)
__global__ void __launch_bounds__(VEC_THREADS) k_true_residual(int64_t n, const double *__restrict__ b,
                                                               const double *__restrict__ ap,
                                                               double *partials, SolverState *st) {
    double v[1] = {0.0};
    FG_VEC4_LOOP(q, n) {
        const V4<double> bv = ld4(b, q), av = ld4(ap, q);
        FG_K4 {
            const double s = bv.a[k] - av.a[k];
            v[0] += s * s;
        }
    }
    double tot[1];
    if (grid_sum<1>(v, partials, st, tot) && threadIdx.x == 0)
        st->tmp[0] = st->bnorm == 0.0 ? 0.0 : sqrt(tot[0]) / st->bnorm;
}

// Deterministic splitmix64 start vector in [-1,1) on the plain DOF index
// (same sequence as the oracle); pads stay zero.
__device__ __forceinline__ double hash_unit(uint64_t i) {
    uint64_t z = i + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z = z ^ (z >> 31);
    return (double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

__global__ void __launch_bounds__(VEC_THREADS) k_hash_vector(const Grid g, double *__restrict__ v,
                                                             double *partials, SolverState *st) {
    const int64_t n = (int64_t)g.NIp * g.NJ * g.NK;
    double acc[1] = {0.0};
    FG_VEC_LOOP(i, n) {
        const int I = (int)(i % g.NIp);
        const int64_t row = i / g.NIp;
        double s = 0.0;
        if (I < g.NI) s = hash_unit((uint64_t)(row * g.NI + I));
        v[i] = s;
        acc[0] += s * s;
    }
    double tot[1];
    if (grid_sum<1>(acc, partials, st, tot) && threadIdx.x == 0) st->rho = sqrt(tot[0]);
}

// v /= rho (if rho > 1e-14)
__global__ void __launch_bounds__(VEC_THREADS) k_scale_by_rho(int64_t n, const double *__restrict__ w,
                                                              double *__restrict__ v,
                                                              const SolverState *st) {
    const double rho = st->rho;
    if (!(rho > 1e-14)) return;
    const double inv = 1.0 / rho;
    FG_VEC4_LOOP(q, n) {
        V4<double> wv = ld4(w, q);
        FG_K4 wv.a[k] *= inv;
        st4(v, q, wv);
    }
}

// w = dinv * w ; rho = ||w||
__global__ void __launch_bounds__(VEC_THREADS) k_dinv_norm(int64_t n, double *__restrict__ w,
                                                           const double *__restrict__ dinv,
                                                           double *partials, SolverState *st) {
    double acc[1] = {0.0};
    FG_VEC4_LOOP(q, n) {
        V4<double> wv = ld4(w, q);
        const V4<double> dv = ld4(dinv, q);
        FG_K4 {
            wv.a[k] *= dv.a[k];
            acc[0] += wv.a[k] * wv.a[k];
        }
        st4(w, q, wv);
    }
    double tot[1];
    if (grid_sum<1>(acc, partials, st, tot) && threadIdx.x == 0) st->rho = sqrt(tot[0]);
}

// dinv = 1/d if |d| > 1e-30 else 1 on real DOFs (par_solver.rs:271-274); pads 0
template <typename T>
__global__ void __launch_bounds__(VEC_THREADS) k_invert_diag(const Grid g, const double *__restrict__ d,
                                                             T *__restrict__ dinv) {
    const int64_t n = (int64_t)g.NIp * g.NJ * g.NK;
    FG_VEC_LOOP(i, n) {
        const int I = (int)(i % g.NIp);
        const double di = d[i];
        dinv[i] = (T)((I < g.NI) ? (fabs(di) > 1e-30 ? 1.0 / di : 1.0) : 0.0);
    }
}

// ---- FP64 iterative refinement around an FP32 inner solve ----------------

// r = b - ap (FP64); st->rr = ||r||^2, st->res = ||r|| / bnorm; on the first
// call (init) also st->bnorm = ||b||.  Sets done/converged against rtol/atol.
__global__ void __launch_bounds__(VEC_THREADS) k_ir_residual(int64_t n, const double *__restrict__ b,
                                                             const double *__restrict__ ap,
                                                             double *__restrict__ r, double *partials,
                                                             SolverState *st, int init) {
    double v[2] = {0.0, 0.0};
    FG_VEC4_LOOP(q, n) {
        const V4<double> bv = ld4(b, q), av = ld4(ap, q);
        V4<double> rv;
        FG_K4 {
            rv.a[k] = bv.a[k] - av.a[k];
            v[0] += rv.a[k] * rv.a[k];
            if (init) v[1] += bv.a[k] * bv.a[k];
        }
        st4(r, q, rv);
    }
    double tot[2];
    if (grid_sum<2>(v, partials, st, tot) && threadIdx.x == 0) {
        if (init) {
            st->bb = tot[1];
            st->bnorm = sqrt(tot[1]);
            st->iter = 0;
            st->converged = 0;
            st->breakdown = 0;
            st->done = 0;
        }
        st->rr = tot[0];
        const double rn = sqrt(tot[0]);
        st->res = st->bnorm == 0.0 ? 0.0 : rn / st->bnorm;
        if (st->bnorm < 1e-30 || st->res < st->rtol || rn < st->atol) {
            st->converged = 1;
            st->done = 1;
        }
    }
}

// r32 = r / ||r|| (the inner solve sees a unit right-hand side)
__global__ void __launch_bounds__(VEC_THREADS) k_ir_to_f32(int64_t n, const double *__restrict__ r,
                                                           float *__restrict__ r32,
                                                           const SolverState *st) {
    const double s = st->rr > 0.0 ? 1.0 / sqrt(st->rr) : 0.0;
    FG_VEC4_LOOP(q, n) {
        const V4<double> rv = ld4(r, q);
        V4<float> o;
        FG_K4 o.a[k] = (float)(rv.a[k] * s);
        st4(r32, q, o);
    }
}

// x += ||r|| * e   (FP64 solution update)
__global__ void __launch_bounds__(VEC_THREADS) k_ir_update(int64_t n, double *__restrict__ x,
                                                           const float *__restrict__ e,
                                                           const SolverState *st) {
    const double s = sqrt(st->rr);
    FG_VEC4_LOOP(q, n) {
        V4<double> xv = ld4(x, q);
        const V4<float> ev = ld4(e, q);
        FG_K4 xv.a[k] += s * (double)ev.a[k];
        st4(x, q, xv);
    }
}

// FP32 copy of an FP64 vector
__global__ void __launch_bounds__(VEC_THREADS) k_to_f32(int64_t n, const double *__restrict__ a,
                                                        float *__restrict__ b) {
    FG_VEC_LOOP(i, n) b[i] = (float)a[i];
}

// Rows of `w` values from a layout of row pitch `sp` to one of pitch `dp` (the
// plain <-> padded native layouts): one warp per row, lanes across the row.
// On the SMs, so that the copy engines stay free for the PCIe transfers of a
// host-memory apply.
template <typename T>
__global__ void __launch_bounds__(256) k_repitch(const T *__restrict__ src, int64_t sp, T *__restrict__ dst,
                                                 int64_t dp, int w, int64_t rows) {
    const int lane = threadIdx.x & 31;
    const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t r = wid; r < rows; r += nw) {
        const T *s = src + r * sp;
        T *d = dst + r * dp;
        for (int c = lane; c < w; c += 32) d[c] = __ldg(s + c);
    }
}

// ---- mixed-precision PCG with reliable updates -----------------------------
// FP32 iterates (x_lo: correction since the last update, r_lo, p, z), FP64
// solution x and FP64 dot products.  When ||r_lo|| has dropped by `delta`
// since the last update (or meets rtol, or max_iter is reached) the update is
// "reliable": x += x_lo, x_lo = 0, r_lo = b - A x recomputed in FP64.  The
// search direction p is kept, so the Krylov space is not thrown away.

// x_lo += alpha p ; r_lo -= alpha ap ; rr ; sets trigger
__global__ void __launch_bounds__(VEC_THREADS) k_rel_step(int64_t n, float *__restrict__ xlo,
                                                          float *__restrict__ r,
                                                          const float *__restrict__ p,
                                                          const float *__restrict__ ap,
                                                          double *partials, SolverState *st) {
    if (st->done) return;
    const float alpha = (float)st->alpha;
    double v[1] = {0.0};
    FG_VEC4_LOOP(q, n) {
        V4<float> xv = ld4(xlo, q), rv = ld4(r, q);
        const V4<float> pv = ld4(p, q), av = ld4(ap, q);
        FG_K4 {
            xv.a[k] += alpha * pv.a[k];
            rv.a[k] = rv.a[k] - alpha * av.a[k];
            v[0] += (double)rv.a[k] * (double)rv.a[k];
        }
        st4(xlo, q, xv);
        st4(r, q, rv);
    }
    double tot[1];
    if (grid_sum<1>(v, partials, st, tot) && threadIdx.x == 0) {
        st->iter += 1;
        st->rr = tot[0];
        const double rn = sqrt(tot[0]);
        const int trig = (rn < st->delta * st->maxr) || (rn / st->bnorm < st->rtol) ||
                         (rn < st->atol) || (st->iter >= st->max_iter);
        st->trigger = trig;
        st->skip_rel = !trig;
    }
}

// reliable update, part 1: x += x_lo ; x_lo = 0
__global__ void __launch_bounds__(VEC_THREADS) k_rel_xupdate(int64_t n, double *__restrict__ x,
                                                             float *__restrict__ xlo,
                                                             const SolverState *st) {
    if (!st->trigger) return;
    FG_VEC4_LOOP(q, n) {
        V4<double> xv = ld4(x, q);
        const V4<float> lv = ld4(xlo, q);
        FG_K4 xv.a[k] += (double)lv.a[k];
        st4(x, q, xv);
        st4(xlo, q, V4<float>{{0.0f, 0.0f, 0.0f, 0.0f}});
    }
}

// reliable update, part 2 (after ap = A x in FP64): r_lo = b - ap ; true residual
// check; on init also bnorm.  init also runs when trigger is clear.
__global__ void __launch_bounds__(VEC_THREADS) k_rel_residual(int64_t n, const double *__restrict__ b,
                                                              const double *__restrict__ ap,
                                                              float *__restrict__ r,
                                                              double *partials, SolverState *st,
                                                              int init) {
    if (!init && !st->trigger) return;
    double v[2] = {0.0, 0.0};
    FG_VEC4_LOOP(q, n) {
        const V4<double> bv = ld4(b, q), av = ld4(ap, q);
        V4<float> rv;
        FG_K4 {
            const double ri = bv.a[k] - av.a[k];
            rv.a[k] = (float)ri;
            v[0] += ri * ri;
            if (init) v[1] += bv.a[k] * bv.a[k];
        }
        st4(r, q, rv);
    }
    double tot[2];
    if (grid_sum<2>(v, partials, st, tot) && threadIdx.x == 0) {
        if (init) {
            st->bb = tot[1];
            st->bnorm = sqrt(tot[1]);
            st->iter = 0;
            st->converged = 0;
            st->breakdown = 0;
            st->done = 0;
            st->tmp[1] = 0.0;
        } else {
            st->tmp[1] += 1.0;  // reliable updates done
        }
        const double rn = sqrt(tot[0]);
        st->rr = tot[0];
        st->maxr = rn;
        st->res = st->bnorm == 0.0 ? 0.0 : rn / st->bnorm;
        st->trigger = 0;
        st->skip_rel = 1;
        if (st->bnorm < 1e-30 || st->res < st->rtol || rn < st->atol) {
            st->converged = 1;
            st->done = 1;
        } else if (st->iter >= st->max_iter) {
            st->done = 1;
        }
    }
}

// z = dinv r ; rz_new = r.z ; beta (init: rz only)
template <typename T>
__global__ void __launch_bounds__(VEC_THREADS) k_jacobi_rz(int64_t n, const T *__restrict__ r,
                                                           const T *__restrict__ dinv,
                                                           T *__restrict__ z, double *partials,
                                                           SolverState *st, int init) {
    if (st->done) return;
    double v[1] = {0.0};
    FG_VEC4_LOOP(q, n) {
        const V4<T> rv = ld4(r, q), dv = ld4(dinv, q);
        V4<T> zv;
        FG_K4 {
            zv.a[k] = dv.a[k] * rv.a[k];
            v[0] += (double)rv.a[k] * (double)zv.a[k];
        }
        st4(z, q, zv);
    }
    double tot[1];
    if (grid_sum<1>(v, partials, st, tot) && threadIdx.x == 0) {
        if (!init) st->beta = tot[0] / st->rz;
        st->rz = tot[0];
    }
}

// out = a x + b y   (FP64; SDIRK stage combinations)
__global__ void __launch_bounds__(VEC_THREADS) k_lincomb2(int64_t n, double *__restrict__ out, double a,
                                                          const double *__restrict__ x, double b,
                                                          const double *__restrict__ y) {
    FG_VEC4_LOOP(q, n) {
        const V4<double> xv = ld4(x, q), yv = ld4(y, q);
        V4<double> o;
        FG_K4 o.a[k] = a * xv.a[k] + b * yv.a[k];
        st4(out, q, o);
    }
}

// ---- batched solves: blockIdx.y = instance ---------------------------------
// Per-instance pointers, state and Chebyshev coefficients; reductions use the
// instance's own partials and ticket (grid_sum over gridDim.x blocks).
constexpr int BATCH_MAXK = 16;
struct BatchVec {
    int64_t n;
    double *x64, *b64, *ap64;
    float *r, *z, *p, *ap, *e, *cres, *cd, *ct;
    const float *dinv;
    double *partials;
    SolverState *st;
    double inv_theta;
    double c1[BATCH_MAXK], c2[BATCH_MAXK];
};

__global__ void __launch_bounds__(VEC_THREADS) kb_pap(const BatchVec *bv) {
    const BatchVec &B = bv[blockIdx.y];
    SolverState *st = B.st;
    if (st->done) return;
    double v[1] = {0.0};
    FG_VEC4_LOOP(q, B.n) {
        const V4<float> pv = ld4(B.p, q), av = ld4(B.ap, q);
        FG_K4 v[0] += (double)pv.a[k] * (double)av.a[k];
    }
    double tot[1];
    if (grid_sum<1>(v, B.partials, st, tot) && threadIdx.x == 0) {
        st->pap = tot[0];
        if (fabs(tot[0]) < 1e-30) {
            st->breakdown = 1;
            st->done = 1;
            st->skip_rel = 1;
        } else {
            st->alpha = st->rz / tot[0];
        }
    }
}

__global__ void __launch_bounds__(VEC_THREADS) kb_rel_step(const BatchVec *bv) {
    const BatchVec &B = bv[blockIdx.y];
    SolverState *st = B.st;
    if (st->done) return;
    const float alpha = (float)st->alpha;
    double v[1] = {0.0};
    FG_VEC4_LOOP(q, B.n) {
        V4<float> xv = ld4(B.e, q), rv = ld4(B.r, q);
        const V4<float> pv = ld4(B.p, q), av = ld4(B.ap, q);
        FG_K4 {
            xv.a[k] += alpha * pv.a[k];
            rv.a[k] = rv.a[k] - alpha * av.a[k];
            v[0] += (double)rv.a[k] * (double)rv.a[k];
        }
        st4(B.e, q, xv);
        st4(B.r, q, rv);
    }
    double tot[1];
    if (grid_sum<1>(v, B.partials, st, tot) && threadIdx.x == 0) {
        st->iter += 1;
        st->rr = tot[0];
        const double rn = sqrt(tot[0]);
        const int trig = (rn < st->delta * st->maxr) || (rn / st->bnorm < st->rtol) ||
                         (rn < st->atol) || (st->iter >= st->max_iter);
        st->trigger = trig;
        st->skip_rel = !trig;
    }
}

__global__ void __launch_bounds__(VEC_THREADS) kb_rel_xupdate(const BatchVec *bv) {
    const BatchVec &B = bv[blockIdx.y];
    if (!B.st->trigger) return;
    FG_VEC4_LOOP(q, B.n) {
        V4<double> xv = ld4(B.x64, q);
        const V4<float> lv = ld4(B.e, q);
        FG_K4 xv.a[k] += (double)lv.a[k];
        st4(B.x64, q, xv);
        st4(B.e, q, V4<float>{{0.0f, 0.0f, 0.0f, 0.0f}});
    }
}

__global__ void __launch_bounds__(VEC_THREADS) kb_rel_residual(const BatchVec *bv, int init) {
    const BatchVec &B = bv[blockIdx.y];
    SolverState *st = B.st;
    if (!init && !st->trigger) return;
    double v[2] = {0.0, 0.0};
    FG_VEC4_LOOP(q, B.n) {
        const V4<double> bb = ld4(B.b64, q), av = ld4(B.ap64, q);
        V4<float> rv;
        FG_K4 {
            const double ri = bb.a[k] - av.a[k];
            rv.a[k] = (float)ri;
            v[0] += ri * ri;
            if (init) v[1] += bb.a[k] * bb.a[k];
        }
        st4(B.r, q, rv);
    }
    double tot[2];
    if (grid_sum<2>(v, B.partials, st, tot) && threadIdx.x == 0) {
        if (init) {
            st->bb = tot[1];
            st->bnorm = sqrt(tot[1]);
            st->iter = 0;
            st->converged = 0;
            st->breakdown = 0;
            st->done = 0;
            st->tmp[1] = 0.0;
        } else {
            st->tmp[1] += 1.0;
        }
        const double rn = sqrt(tot[0]);
        st->rr = tot[0];
        st->maxr = rn;
        st->res = st->bnorm == 0.0 ? 0.0 : rn / st->bnorm;
        st->trigger = 0;
        st->skip_rel = 1;
        if (st->bnorm < 1e-30 || st->res < st->rtol || rn < st->atol) {
            st->converged = 1;
            st->done = 1;
        } else if (st->iter >= st->max_iter) {
            st->done = 1;
        }
    }
}

__global__ void __launch_bounds__(VEC_THREADS) kb_cheb_first(const BatchVec *bv) {
    const BatchVec &B = bv[blockIdx.y];
    if (B.st->done) return;
    const float it = (float)B.inv_theta;
    FG_VEC4_LOOP(q, B.n) {
        const V4<float> rv = ld4(B.r, q), dv = ld4(B.dinv, q);
        V4<float> sv, dd;
        FG_K4 {
            sv.a[k] = dv.a[k] * rv.a[k];
            dd.a[k] = sv.a[k] * it;
        }
        st4(B.cres, q, sv);
        st4(B.cd, q, dd);
        st4(B.z, q, dd);
    }
}

// last: the final sweep, whose residual and d are not needed afterwards (two
// stores fewer; z is the same)
__global__ void __launch_bounds__(VEC_THREADS) kb_cheb_step(const BatchVec *bv, int s, int last) {
    const BatchVec &B = bv[blockIdx.y];
    if (B.st->done) return;
    const float a1 = (float)B.c1[s], a2 = (float)B.c2[s];
    FG_VEC4_LOOP(q, B.n) {
        const V4<float> tv = ld4(B.ct, q), dv = ld4(B.dinv, q);
        V4<float> sv = ld4(B.cres, q), dd = ld4(B.cd, q), zv = ld4(B.z, q);
        FG_K4 {
            sv.a[k] = sv.a[k] - dv.a[k] * tv.a[k];
            dd.a[k] = a1 * dd.a[k] + a2 * sv.a[k];
            zv.a[k] += dd.a[k];
        }
        if (!last) {
            st4(B.cres, q, sv);
            st4(B.cd, q, dd);
        }
        st4(B.z, q, zv);
    }
}

// jacobi: z = dinv r first; then rz_new = r.z, beta (init: rz only)
__global__ void __launch_bounds__(VEC_THREADS) kb_rz(const BatchVec *bv, int init, int jacobi) {
    const BatchVec &B = bv[blockIdx.y];
    SolverState *st = B.st;
    if (st->done) return;
    double v[1] = {0.0};
    FG_VEC4_LOOP(q, B.n) {
        const V4<float> rv = ld4(B.r, q);
        V4<float> zv;
        if (jacobi) {
            const V4<float> dv = ld4(B.dinv, q);
            FG_K4 zv.a[k] = dv.a[k] * rv.a[k];
            st4(B.z, q, zv);
        } else {
            zv = ld4(B.z, q);
        }
        FG_K4 v[0] += (double)rv.a[k] * (double)zv.a[k];
    }
    double tot[1];
    if (grid_sum<1>(v, B.partials, st, tot) && threadIdx.x == 0) {
        if (!init) st->beta = tot[0] / st->rz;
        st->rz = tot[0];
    }
}

__global__ void __launch_bounds__(VEC_THREADS) kb_pupdate(const BatchVec *bv, int init) {
    const BatchVec &B = bv[blockIdx.y];
    if (B.st->done) return;
    const float beta = init ? 0.0f : (float)B.st->beta;
    FG_VEC4_LOOP(q, B.n) {
        const V4<float> zv = ld4(B.z, q);
        V4<float> pv = init ? zv : ld4(B.p, q);  // first direction: p is not read
        if (!init) {
            FG_K4 pv.a[k] = zv.a[k] + beta * pv.a[k];
        }
        st4(B.p, q, pv);
    }
}

__global__ void __launch_bounds__(VEC_THREADS) kb_zero_e(const BatchVec *bv) {
    const BatchVec &B = bv[blockIdx.y];
    FG_VEC4_LOOP(q, B.n) st4(B.e, q, V4<float>{{0.0f, 0.0f, 0.0f, 0.0f}});
}

__global__ void __launch_bounds__(VEC_THREADS) kb_true_residual(const BatchVec *bv) {
    const BatchVec &B = bv[blockIdx.y];
    SolverState *st = B.st;
    double v[1] = {0.0};
    FG_VEC4_LOOP(q, B.n) {
        const V4<double> bb = ld4(B.b64, q), av = ld4(B.ap64, q);
        FG_K4 {
            const double s = bb.a[k] - av.a[k];
            v[0] += s * s;
        }
    }
    double tot[1];
    if (grid_sum<1>(v, B.partials, st, tot) && threadIdx.x == 0)
        st->tmp[0] = st->bnorm == 0.0 ? 0.0 : sqrt(tot[0]) / st->bnorm;
}

// st->tmp[2] = ||v|| (FP64)
__global__ void __launch_bounds__(VEC_THREADS) k_norm_tmp(int64_t n, const double *__restrict__ v,
                                                          double *partials, SolverState *st) {
    double a[1] = {0.0};
    FG_VEC4_LOOP(q, n) {
        const V4<double> x = ld4(v, q);
        FG_K4 a[0] += x.a[k] * x.a[k];
    }
    double tot[1];
    if (grid_sum<1>(a, partials, st, tot) && threadIdx.x == 0) st->tmp[2] = sqrt(tot[0]);
}

// v *= 1/tmp[2] (inverse = 1) or v *= tmp[2]; no-op when tmp[2] == 0
__global__ void __launch_bounds__(VEC_THREADS) k_scale_tmp(int64_t n, double *__restrict__ v,
                                                           const SolverState *st, int inverse) {
    const double s = st->tmp[2];
    if (!(s > 0.0)) return;
    const double f = inverse ? 1.0 / s : s;
    FG_VEC4_LOOP(q, n) {
        V4<double> x = ld4(v, q);
        FG_K4 x.a[k] *= f;
        st4(v, q, x);
    }
}

// energy terms of a coarse correction c:  st->tmp[0] = c . (A c),
// st->tmp[1] = c . r;  ac <- A c - r
__global__ void __launch_bounds__(VEC_THREADS) k_energy_terms(int64_t n, const double *__restrict__ c,
                                                              double *__restrict__ ac, const double *__restrict__ r,
                                                              double *partials, SolverState *st) {
    double a[2] = {0.0, 0.0};
    FG_VEC4_LOOP(q, n) {
        const V4<double> cv = ld4(c, q), rv = ld4(r, q);
        V4<double> av = ld4(ac, q);
        FG_K4 {
            a[0] += cv.a[k] * av.a[k];
            a[1] += cv.a[k] * rv.a[k];
            av.a[k] -= rv.a[k];
        }
        st4(ac, q, av);
    }
    double tot[2];
    if (grid_sum<2>(a, partials, st, tot) && threadIdx.x == 0) {
        st->tmp[0] = tot[0];
        st->tmp[1] = tot[1];
    }
}

// ---- flexible CG (Notay's FCG with one stored direction) -------------------
// beta = -(z . A p_old) / (p_old . A p_old)  (0 on init);  then p = z + beta p
template <typename T>
__global__ void __launch_bounds__(VEC_THREADS) k_fcg_zap(int64_t n, const T *__restrict__ z,
                                                         const T *__restrict__ ap, double *partials,
                                                         SolverState *st, int init) {
    if (st->done) return;
    double v[1] = {0.0};
    if (!init) {
        FG_VEC4_LOOP(q, n) {
            const V4<T> zv = ld4(z, q), av = ld4(ap, q);
            FG_K4 v[0] += (double)zv.a[k] * (double)av.a[k];
        }
    }
    double tot[1];
    if (grid_sum<1>(v, partials, st, tot) && threadIdx.x == 0)
        st->beta = init ? 0.0 : -tot[0] / st->pap;
}

// p = z + beta p (init: p = z) and rz = p . r in one pass: the values of
// k_pcg_pupdate followed by a separate p . r pass (same loop order, same sums),
// one vector pass and one launch fewer.  rz is the FCG step numerator (alpha =
// rz / pap in k_pcg_pap)
template <typename T>
__global__ void __launch_bounds__(VEC_THREADS) k_fcg_pupdate_pr(int64_t n, const T *__restrict__ z,
                                                                T *__restrict__ p,
                                                                const T *__restrict__ r, double *partials,
                                                                SolverState *st, int init) {
    if (st->done) return;
    const T beta = init ? T(0) : (T)st->beta;
    double v[1] = {0.0};
    FG_VEC4_LOOP(q, n) {
        const V4<T> zv = ld4(z, q), rv = ld4(r, q);
        V4<T> pv = init ? zv : ld4(p, q);  // first direction: p is not read
        if (!init) {
            FG_K4 pv.a[k] = zv.a[k] + beta * pv.a[k];
        }
        st4(p, q, pv);
        FG_K4 v[0] += (double)pv.a[k] * (double)rv.a[k];
    }
    double tot[1];
    if (grid_sum<1>(v, partials, st, tot) && threadIdx.x == 0) st->rz = tot[0];
}

}  // namespace fg

// ---- steps of a solve whose dots are completed outside the library ----------
// (the sharded PCG: each rank reduces over the DOFs it owns, the caller's
// allreduce adds the ranks' partial sums, and the scalars stay on the
// device).  The owned DOFs are the prefix [0, n_own) of the local vector (a
// multiple of 4).  Same deterministic block-order sums as above.
namespace fg {
struct VecPairs {
    const double *a[3];
    const double *b[3];
};

// out[j] = sum_{i < n_own} a_j[i] b_j[i], j < NV
template <int NV>
__global__ void __launch_bounds__(VEC_THREADS) k_sh_dots(int64_t n_own, const VecPairs P, double *partials,
                                                         SolverState *st, double *out) {
    double v[NV];
#pragma unroll
    for (int j = 0; j < NV; ++j) v[j] = 0.0;
    FG_VEC4_LOOP(q, n_own) {
#pragma unroll
        for (int j = 0; j < NV; ++j) {
            const V4<double> av = ld4(P.a[j], q), bv = ld4(P.b[j], q);
            FG_K4 v[j] += av.a[k] * bv.a[k];
        }
    }
    double tot[NV];
    if (grid_sum<NV>(v, partials, st, tot) && threadIdx.x == 0)
#pragma unroll
        for (int j = 0; j < NV; ++j) out[j] = tot[j];
}

// alpha = s[0] / s[1] (r.z / p.Ap after the allreduce); x += alpha p,
// r -= alpha Ap, z = dinv r on the whole local vector; out = (r.r, r.z) over
// the owned prefix
__global__ void __launch_bounds__(VEC_THREADS) k_sh_update(int64_t n, int64_t n_own, double *__restrict__ x,
                                                           double *__restrict__ r, const double *__restrict__ p,
                                                           const double *__restrict__ ap,
                                                           const double *__restrict__ dinv, double *__restrict__ z,
                                                           const double *s, double *partials, SolverState *st,
                                                           double *out) {
    const double alpha = s[0] / s[1];
    double v[2] = {0.0, 0.0};
    FG_VEC4_LOOP(q, n) {
        V4<double> xv = ld4(x, q), rv = ld4(r, q), zv;
        const V4<double> pv = ld4(p, q), av = ld4(ap, q), dv = ld4(dinv, q);
        FG_K4 {
            xv.a[k] += alpha * pv.a[k];
            rv.a[k] -= alpha * av.a[k];
            zv.a[k] = dv.a[k] * rv.a[k];
        }
        st4(x, q, xv);
        st4(r, q, rv);
        st4(z, q, zv);
        if (4 * q < n_own) {
            FG_K4 {
                v[0] += rv.a[k] * rv.a[k];
                v[1] += rv.a[k] * zv.a[k];
            }
        }
    }
    double tot[2];
    if (grid_sum<2>(v, partials, st, tot) && threadIdx.x == 0) {
        out[0] = tot[0];
        out[1] = tot[1];
    }
}

// p = z + (num / den) p
__global__ void __launch_bounds__(VEC_THREADS) k_sh_pupdate(int64_t n, const double *__restrict__ z,
                                                            double *__restrict__ p, const double *num,
                                                            const double *den) {
    const double beta = *num / *den;
    FG_VEC4_LOOP(q, n) {
        const V4<double> zv = ld4(z, q);
        V4<double> pv = ld4(p, q);
        FG_K4 pv.a[k] = zv.a[k] + beta * pv.a[k];
        st4(p, q, pv);
    }
}
}  // namespace fg
