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
    int iter, done, converged, breakdown, max_iter;
    unsigned int ticket;
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

// r = b - ap; z = dinv r (jacobi) ; p = z ; rz = r.z ; bb = b.b
__global__ void __launch_bounds__(VEC_THREADS) k_pcg_init(int64_t n, const double *__restrict__ b,
                                                          const double *__restrict__ ap,
                                                          const double *__restrict__ dinv,
                                                          double *__restrict__ r, double *__restrict__ z,
                                                          double *__restrict__ p, int jacobi,
                                                          double *partials, SolverState *st) {
    double v[2] = {0.0, 0.0};
    FG_VEC_LOOP(i, n) {
        const double ri = b[i] - ap[i];
        r[i] = ri;
        v[1] += b[i] * b[i];
        if (jacobi) {
            const double zi = dinv[i] * ri;
            z[i] = zi;
            p[i] = zi;
            v[0] += ri * zi;
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
        if (st->bnorm < 1e-30) {
            st->converged = 1;
            st->done = 1;
            st->res = 0.0;
        }
    }
}

// pap = p.ap ; alpha = rz / pap  (breakdown if |pap| < 1e-30)
__global__ void __launch_bounds__(VEC_THREADS) k_pcg_pap(int64_t n, const double *__restrict__ p,
                                                         const double *__restrict__ ap,
                                                         double *partials, SolverState *st) {
    if (st->done) return;
    double v[1] = {0.0};
    FG_VEC_LOOP(i, n) v[0] += p[i] * ap[i];
    double tot[1];
    if (grid_sum<1>(v, partials, st, tot) && threadIdx.x == 0) {
        st->pap = tot[0];
        if (fabs(tot[0]) < 1e-30) {
            st->breakdown = 1;
            st->done = 1;
        } else {
            st->alpha = st->rz / tot[0];
        }
    }
}

// x += alpha p ; r -= alpha ap ; [jacobi: z = dinv r, rz_new] ; rr ; convergence
__global__ void __launch_bounds__(VEC_THREADS) k_pcg_update(int64_t n, double *__restrict__ x,
                                                            double *__restrict__ r,
                                                            const double *__restrict__ p,
                                                            const double *__restrict__ ap,
                                                            const double *__restrict__ dinv,
                                                            double *__restrict__ z, int jacobi,
                                                            double *partials, SolverState *st) {
    if (st->done) return;
    const double alpha = st->alpha;
    double v[2] = {0.0, 0.0};
    FG_VEC_LOOP(i, n) {
        x[i] += alpha * p[i];
        const double ri = r[i] - alpha * ap[i];
        r[i] = ri;
        v[0] += ri * ri;
        if (jacobi) {
            const double zi = dinv[i] * ri;
            z[i] = zi;
            v[1] += ri * zi;
        }
    }
    double tot[2];
    if (grid_sum<2>(v, partials, st, tot) && threadIdx.x == 0) {
        st->iter += 1;
        st->rr = tot[0];
        const double rn = sqrt(tot[0]);
        st->res = rn / st->bnorm;
        if (st->res < st->rtol || rn < st->atol) {
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

// rz_new = r.z ; beta = rz_new / rz ; rz = rz_new   (non-Jacobi preconditioners)
__global__ void __launch_bounds__(VEC_THREADS) k_pcg_rz(int64_t n, const double *__restrict__ r,
                                                        const double *__restrict__ z,
                                                        double *partials, SolverState *st, int init) {
    if (st->done) return;
    double v[1] = {0.0};
    FG_VEC_LOOP(i, n) v[0] += r[i] * z[i];
    double tot[1];
    if (grid_sum<1>(v, partials, st, tot) && threadIdx.x == 0) {
        if (!init) st->beta = tot[0] / st->rz;
        st->rz = tot[0];
    }
}

// p = z + beta p   (init: p = z)
__global__ void __launch_bounds__(VEC_THREADS) k_pcg_pupdate(int64_t n, const double *__restrict__ z,
                                                             double *__restrict__ p,
                                                             const SolverState *st, int init) {
    if (st->done) return;
    const double beta = init ? 0.0 : st->beta;
    FG_VEC_LOOP(i, n) p[i] = z[i] + beta * p[i];
}

// Chebyshev sweep 1 from zero: res = dinv r ; d = res / theta ; z = d
__global__ void __launch_bounds__(VEC_THREADS) k_cheb_first(int64_t n, const double *__restrict__ r,
                                                            const double *__restrict__ dinv,
                                                            double *__restrict__ res,
                                                            double *__restrict__ d,
                                                            double *__restrict__ z, double inv_theta,
                                                            const SolverState *st) {
    if (st && st->done) return;
    FG_VEC_LOOP(i, n) {
        const double s = dinv[i] * r[i];
        res[i] = s;
        const double di = s * inv_theta;
        d[i] = di;
        z[i] = di;
    }
}

// Chebyshev sweep: res -= dinv t ; d = c1 d + c2 res ; z += d
__global__ void __launch_bounds__(VEC_THREADS) k_cheb_step(int64_t n, const double *__restrict__ t,
                                                           const double *__restrict__ dinv,
                                                           double *__restrict__ res,
                                                           double *__restrict__ d,
                                                           double *__restrict__ z, double c1,
                                                           double c2, const SolverState *st) {
    if (st && st->done) return;
    FG_VEC_LOOP(i, n) {
        const double s = res[i] - dinv[i] * t[i];
        res[i] = s;
        const double di = c1 * d[i] + c2 * s;
        d[i] = di;
        z[i] += di;
    }
}

// ||b - ap|| / bnorm into st->tmp[0] (true residual)
__global__ void __launch_bounds__(VEC_THREADS) k_true_residual(int64_t n, const double *__restrict__ b,
                                                               const double *__restrict__ ap,
                                                               double *partials, SolverState *st) {
    double v[1] = {0.0};
    FG_VEC_LOOP(i, n) {
        const double s = b[i] - ap[i];
        v[0] += s * s;
    }
    double tot[1];
    if (grid_sum<1>(v, partials, st, tot) && threadIdx.x == 0)
        st->tmp[0] = st->bnorm > 0.0 ? sqrt(tot[0]) / st->bnorm : 0.0;
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
    FG_VEC_LOOP(i, n) v[i] = w[i] * inv;
}

// w = dinv * w ; rho = ||w||
__global__ void __launch_bounds__(VEC_THREADS) k_dinv_norm(int64_t n, double *__restrict__ w,
                                                           const double *__restrict__ dinv,
                                                           double *partials, SolverState *st) {
    double acc[1] = {0.0};
    FG_VEC_LOOP(i, n) {
        const double s = dinv[i] * w[i];
        w[i] = s;
        acc[0] += s * s;
    }
    double tot[1];
    if (grid_sum<1>(acc, partials, st, tot) && threadIdx.x == 0) st->rho = sqrt(tot[0]);
}

// dinv = 1/d if |d| > 1e-30 else 1 on real DOFs (par_solver.rs:271-274); pads 0
__global__ void __launch_bounds__(VEC_THREADS) k_invert_diag(const Grid g, const double *__restrict__ d,
                                                             double *__restrict__ dinv) {
    const int64_t n = (int64_t)g.NIp * g.NJ * g.NK;
    FG_VEC_LOOP(i, n) {
        const int I = (int)(i % g.NIp);
        const double di = d[i];
        dinv[i] = (I < g.NI) ? (fabs(di) > 1e-30 ? 1.0 / di : 1.0) : 0.0;
    }
}

}  // namespace fg
