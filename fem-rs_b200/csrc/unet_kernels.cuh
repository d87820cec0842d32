// unet_kernels.cuh -- kernels of the learned coarse correction: a small 3-D
// U-net on the vertex grid coarsened twice from the Q1 DOF grid.
//
// Tensors are dense channels-last BF16 volumes [batch][z][y][x][c] addressed
// through (pointer, channel stride, channel offset) views, so concatenations
// are channel ranges of one buffer.  Arithmetic accumulates in FP32.
//
// conv3_fwd_kernel: 3x3x3 "same" convolution as an implicit GEMM
//   out[v][co] = bias[co] + sum_k W[co][k] * A[v][k],  k = tap*Cin + ci,
//   A[v][k] = in[v + off(tap)][ci] (0 outside the volume),
// on the BF16 tensor cores (mma.sync m16n8k16, FP32 accumulators): a warp owns
// 16 voxels x all output channels; A fragments are gathered straight from the
// input volume (im2col on the fly), B fragments from W[co][Kp] (K padded to a
// multiple of 16 with zeros).  The backward pass w.r.t. the input is the same
// kernel applied to the output gradient with the flipped, transposed weights
// W'[ci][tap][co] = W[co][26-tap][ci].
//
// conv3_wgrad_kernel: dW[co][k] = sum_v dY[v][co] A[v][k] as a GEMM with the
// voxel dimension as K, split over voxel chunks; chunk partials are summed in
// chunk order by conv3_wgrad_reduce (deterministic, no atomics).
#pragma once
#include <cuda_bf16.h>

#include "fg_common.cuh"

namespace fg {

struct Vol {
    int B, Z, Y, X;  // batch and spatial extent
    __host__ __device__ int64_t nvox() const { return (int64_t)B * Z * Y * X; }
};

struct TView {
    __nv_bfloat16 *p;
    int cs, co;  // channel stride (channels per voxel in the buffer), channel offset
};

__device__ __forceinline__ uint32_t ld_bf16x2(const __nv_bfloat16 *p) {
    return *reinterpret_cast<const uint32_t *>(p);
}

__device__ __forceinline__ void mma_bf16_16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0,
                                               uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// voxel index -> coordinates (network volumes hold < 2^31 voxels)
__device__ __forceinline__ void vox_coords(const Vol &V, int64_t v64, int &b, int &z, int &y, int &x) {
    const int v = (int)v64;
    x = v % V.X;
    int t = v / V.X;
    y = t % V.Y;
    t /= V.Y;
    z = t % V.Z;
    b = t / V.Z;
}

// decomposition of a GEMM column k = tap*Cin + ci
struct KCol {
    int ci, dz, dy, dx;
    bool ok;
};
__device__ __forceinline__ KCol kcol(int k, int Cin, int K) {
    KCol c;
    c.ok = k < K;
    const int tap = c.ok ? k / Cin : 0;
    c.ci = k - tap * Cin;
    c.dz = tap / 9 - 1;
    c.dy = (tap / 3) % 3 - 1;
    c.dx = tap % 3 - 1;
    return c;
}

// A[v][k] pair (k even, k+1) for a voxel given by coordinates (valid = in volume)
__device__ __forceinline__ uint32_t gather_pair(const TView &in, const Vol &V, const KCol &c,
                                                bool vvalid, int b, int z, int y, int x) {
    if (!vvalid || !c.ok) return 0u;
    const int zz = z + c.dz, yy = y + c.dy, xx = x + c.dx;
    if (zz < 0 || zz >= V.Z || yy < 0 || yy >= V.Y || xx < 0 || xx >= V.X) return 0u;
    const int64_t vv = (((int64_t)b * V.Z + zz) * V.Y + yy) * V.X + xx;
    return ld_bf16x2(in.p + vv * in.cs + in.co + c.ci);
}

// One tile: 16 voxels x NT*8 output channels, computed by KS warps that split
// the K loop (KS in {1, 2, 4}; a block of 4 warps holds 4/KS tiles) and sum
// their accumulators in shared memory in warp order.  Small volumes use KS = 4
// so that the serial chain of gathers per warp is short.  Cin even,
// Cout = NT*8 <= 80.
template <int NT, int KS>
__global__ void __launch_bounds__(128) conv3_fwd_kernel(const TView in, const Vol V, int Cin,
                                                        const __nv_bfloat16 *__restrict__ W, int Kp,
                                                        const float *__restrict__ bias, TView out,
                                                        int relu) {
    constexpr int TPB = 4 / KS;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tile = warp / KS, part = warp % KS;
    const int gid = lane >> 2, t4 = lane & 3;
    const int64_t nv = V.nvox();
    const int64_t m0 = ((int64_t)blockIdx.x * TPB + tile) * 16;
    const bool active = m0 < nv;
    const int K = 27 * Cin;
    const int64_t v0 = m0 + gid, v1 = m0 + gid + 8;
    int b0, z0, y0, x0, b1, z1, y1, x1;
    vox_coords(V, v0 < nv ? v0 : 0, b0, z0, y0, x0);
    vox_coords(V, v1 < nv ? v1 : 0, b1, z1, y1, x1);
    const bool ok0 = v0 < nv, ok1 = v1 < nv;
    float acc[NT][4];
#pragma unroll
    for (int j = 0; j < NT; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
    if (active) {
#pragma unroll 4
        for (int k0 = part * 16; k0 < Kp; k0 += 16 * KS) {
            const int ka = k0 + t4 * 2, kb = ka + 8;
            const KCol ca = kcol(ka, Cin, K), cb = kcol(kb, Cin, K);
            uint32_t a[4];
            a[0] = gather_pair(in, V, ca, ok0, b0, z0, y0, x0);
            a[1] = gather_pair(in, V, ca, ok1, b1, z1, y1, x1);
            a[2] = gather_pair(in, V, cb, ok0, b0, z0, y0, x0);
            a[3] = gather_pair(in, V, cb, ok1, b1, z1, y1, x1);
#pragma unroll
            for (int j = 0; j < NT; ++j) {
                const __nv_bfloat16 *wr = W + (int64_t)(j * 8 + gid) * Kp;
                mma_bf16_16816(acc[j], a, ld_bf16x2(wr + ka), ld_bf16x2(wr + kb));
            }
        }
    }
    if constexpr (KS > 1) {
        __shared__ float red[TPB * (KS - 1)][NT * 4][32];
        if (part > 0) {
            const int slot = tile * (KS - 1) + part - 1;
#pragma unroll
            for (int j = 0; j < NT; ++j)
#pragma unroll
                for (int e = 0; e < 4; ++e) red[slot][j * 4 + e][lane] = acc[j][e];
        }
        __syncthreads();
        if (part > 0) return;
#pragma unroll
        for (int q = 0; q < KS - 1; ++q)
#pragma unroll
            for (int j = 0; j < NT; ++j)
#pragma unroll
                for (int e = 0; e < 4; ++e) acc[j][e] += red[tile * (KS - 1) + q][j * 4 + e][lane];
    }
    if (!active) return;
#pragma unroll
    for (int j = 0; j < NT; ++j) {
        const int n = j * 8 + t4 * 2;
        const float bb0 = bias ? bias[n] : 0.f, bb1 = bias ? bias[n + 1] : 0.f;
        float r0 = acc[j][0] + bb0, r1 = acc[j][1] + bb1, r2 = acc[j][2] + bb0, r3 = acc[j][3] + bb1;
        if (relu) {
            r0 = fmaxf(r0, 0.f); r1 = fmaxf(r1, 0.f); r2 = fmaxf(r2, 0.f); r3 = fmaxf(r3, 0.f);
        }
        if (ok0)
            *reinterpret_cast<__nv_bfloat162 *>(out.p + v0 * out.cs + out.co + n) = __floats2bfloat162_rn(r0, r1);
        if (ok1)
            *reinterpret_cast<__nv_bfloat162 *>(out.p + v1 * out.cs + out.co + n) = __floats2bfloat162_rn(r2, r3);
    }
}

// Tap-major variant for Cin a multiple of 16 (channel views 4-aligned): the
// neighbour offset and bounds test are computed once per tap and voxel, and
// each 16-channel block is one 8-byte load per voxel and per weight row.  The
// 16 GEMM columns of a block are permuted so that lane t4 holds channels
// 4*t4 .. 4*t4+3 in both operands: fragment columns (2*t4, 2*t4+1) are
// channels 4*t4 + (0, 1) and columns (2*t4+8, 2*t4+9) are 4*t4 + (2, 3).
// The permutation is the same for A and B, so the product is unchanged.
__device__ __forceinline__ uint2 ld_bf16x4(const __nv_bfloat16 *p) {
    return *reinterpret_cast<const uint2 *>(p);
}

template <int NT, int KS>
__global__ void __launch_bounds__(128) conv3_fwd16_kernel(const TView in, const Vol V, int Cin,
                                                          const __nv_bfloat16 *__restrict__ W, int Kp,
                                                          const float *__restrict__ bias, TView out,
                                                          int relu) {
    constexpr int TPB = 4 / KS;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tile = warp / KS, part = warp % KS;
    const int gid = lane >> 2, t4 = lane & 3;
    const int64_t nv = V.nvox();
    const int64_t m0 = ((int64_t)blockIdx.x * TPB + tile) * 16;
    const bool active = m0 < nv;
    const int64_t v0 = m0 + gid, v1 = m0 + gid + 8;
    int b0, z0, y0, x0, b1, z1, y1, x1;
    vox_coords(V, v0 < nv ? v0 : 0, b0, z0, y0, x0);
    vox_coords(V, v1 < nv ? v1 : 0, b1, z1, y1, x1);
    const bool ok0 = v0 < nv, ok1 = v1 < nv;
    float acc[NT][4];
#pragma unroll
    for (int j = 0; j < NT; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
    if (active) {
        const __nv_bfloat16 *wl = W + (int64_t)gid * Kp + 4 * t4;
        for (int tap = part; tap < 27; tap += KS) {
            const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
            const __nv_bfloat16 *p0 = nullptr, *p1 = nullptr;
            {
                const int zz = z0 + dz, yy = y0 + dy, xx = x0 + dx;
                if (ok0 && zz >= 0 && zz < V.Z && yy >= 0 && yy < V.Y && xx >= 0 && xx < V.X)
                    p0 = in.p + ((((int64_t)b0 * V.Z + zz) * V.Y + yy) * V.X + xx) * in.cs + in.co + 4 * t4;
            }
            {
                const int zz = z1 + dz, yy = y1 + dy, xx = x1 + dx;
                if (ok1 && zz >= 0 && zz < V.Z && yy >= 0 && yy < V.Y && xx >= 0 && xx < V.X)
                    p1 = in.p + ((((int64_t)b1 * V.Z + zz) * V.Y + yy) * V.X + xx) * in.cs + in.co + 4 * t4;
            }
            const __nv_bfloat16 *wt = wl + tap * Cin;
#pragma unroll 2
            for (int c0 = 0; c0 < Cin; c0 += 16) {
                const uint2 a0 = p0 ? ld_bf16x4(p0 + c0) : make_uint2(0u, 0u);
                const uint2 a1 = p1 ? ld_bf16x4(p1 + c0) : make_uint2(0u, 0u);
                const uint32_t a[4] = {a0.x, a1.x, a0.y, a1.y};
#pragma unroll
                for (int j = 0; j < NT; ++j) {
                    const uint2 bw = ld_bf16x4(wt + (int64_t)j * 8 * Kp + c0);
                    mma_bf16_16816(acc[j], a, bw.x, bw.y);
                }
            }
        }
    }
    if constexpr (KS > 1) {
        __shared__ float red[TPB * (KS - 1)][NT * 4][32];
        if (part > 0) {
            const int slot = tile * (KS - 1) + part - 1;
#pragma unroll
            for (int j = 0; j < NT; ++j)
#pragma unroll
                for (int e = 0; e < 4; ++e) red[slot][j * 4 + e][lane] = acc[j][e];
        }
        __syncthreads();
        if (part > 0) return;
#pragma unroll
        for (int q = 0; q < KS - 1; ++q)
#pragma unroll
            for (int j = 0; j < NT; ++j)
#pragma unroll
                for (int e = 0; e < 4; ++e) acc[j][e] += red[tile * (KS - 1) + q][j * 4 + e][lane];
    }
    if (!active) return;
#pragma unroll
    for (int j = 0; j < NT; ++j) {
        const int n = j * 8 + t4 * 2;
        const float bb0 = bias ? bias[n] : 0.f, bb1 = bias ? bias[n + 1] : 0.f;
        float r0 = acc[j][0] + bb0, r1 = acc[j][1] + bb1, r2 = acc[j][2] + bb0, r3 = acc[j][3] + bb1;
        if (relu) {
            r0 = fmaxf(r0, 0.f); r1 = fmaxf(r1, 0.f); r2 = fmaxf(r2, 0.f); r3 = fmaxf(r3, 0.f);
        }
        if (ok0)
            *reinterpret_cast<__nv_bfloat162 *>(out.p + v0 * out.cs + out.co + n) = __floats2bfloat162_rn(r0, r1);
        if (ok1)
            *reinterpret_cast<__nv_bfloat162 *>(out.p + v1 * out.cs + out.co + n) = __floats2bfloat162_rn(r2, r3);
    }
}

// Weight gradient partials: block (n-block of 32 columns, voxel chunk), warp =
// m-tile of 16 output channels.  part[chunk][co][Kp] (FP32).
__global__ void __launch_bounds__(128) conv3_wgrad_kernel(const TView in, const Vol V, int Cin,
                                                          const TView dy, int Cout, int Kp, int chunk,
                                                          float *__restrict__ part) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int gid = lane >> 2, t4 = lane & 3;
    const int K = 27 * Cin;
    const int nb0 = blockIdx.x * 32;
    const int mt = warp;  // 16 output channels per warp
    if (mt * 16 >= Cout) return;
    const int64_t nv = V.nvox();
    const int64_t vbeg = (int64_t)blockIdx.y * chunk, vend = min(nv, vbeg + chunk);
    float acc[4][4];
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
    const int co0 = mt * 16 + gid, co1 = co0 + 8;
    for (int64_t vs = vbeg; vs < vend; vs += 16) {
        // A (16 co x 16 voxels): a0 = (co0, v = vs + 2 t4 + {0,1}), a1 = (co1, ...), a2/a3: voxels + 8
        uint32_t a[4];
        __nv_bfloat16 e[8];
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int64_t v = vs + t4 * 2 + q + h * 8;
                const bool ok = v < vend;
                e[h * 4 + q] = (ok && co0 < Cout) ? dy.p[v * dy.cs + dy.co + co0] : __float2bfloat16(0.f);
                e[h * 4 + 2 + q] = (ok && co1 < Cout) ? dy.p[v * dy.cs + dy.co + co1] : __float2bfloat16(0.f);
            }
        a[0] = (uint32_t)__bfloat16_as_ushort(e[0]) | ((uint32_t)__bfloat16_as_ushort(e[1]) << 16);
        a[1] = (uint32_t)__bfloat16_as_ushort(e[2]) | ((uint32_t)__bfloat16_as_ushort(e[3]) << 16);
        a[2] = (uint32_t)__bfloat16_as_ushort(e[4]) | ((uint32_t)__bfloat16_as_ushort(e[5]) << 16);
        a[3] = (uint32_t)__bfloat16_as_ushort(e[6]) | ((uint32_t)__bfloat16_as_ushort(e[7]) << 16);
        // B (16 voxels x 8 columns): b = (k = voxel vs + 2 t4 + {0,1} (+8), n = column nb + gid)
        int vb[4], vz[4], vyy[4], vx[4];
        bool vok[4];
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int64_t v = vs + t4 * 2 + q + h * 8;
                vok[h * 2 + q] = v < vend;
                vox_coords(V, v < vend ? v : vbeg, vb[h * 2 + q], vz[h * 2 + q], vyy[h * 2 + q], vx[h * 2 + q]);
            }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const KCol c = kcol(nb0 + j * 8 + gid, Cin, K);
            uint16_t bv[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                __nv_bfloat16 val = __float2bfloat16(0.f);
                if (vok[u] && c.ok) {
                    const int zz = vz[u] + c.dz, yy = vyy[u] + c.dy, xx = vx[u] + c.dx;
                    if (zz >= 0 && zz < V.Z && yy >= 0 && yy < V.Y && xx >= 0 && xx < V.X) {
                        const int64_t vv = (((int64_t)vb[u] * V.Z + zz) * V.Y + yy) * V.X + xx;
                        val = in.p[vv * in.cs + in.co + c.ci];
                    }
                }
                bv[u] = __bfloat16_as_ushort(val);
            }
            const uint32_t b0 = (uint32_t)bv[0] | ((uint32_t)bv[1] << 16);
            const uint32_t b1 = (uint32_t)bv[2] | ((uint32_t)bv[3] << 16);
            mma_bf16_16816(acc[j], a, b0, b1);
        }
    }
    float *pp = part + (int64_t)blockIdx.y * Cout * Kp;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int n = nb0 + j * 8 + t4 * 2;
        if (n >= Kp) continue;
        if (co0 < Cout) {
            pp[(int64_t)co0 * Kp + n] = acc[j][0];
            pp[(int64_t)co0 * Kp + n + 1] = acc[j][1];
        }
        if (co1 < Cout) {
            pp[(int64_t)co1 * Kp + n] = acc[j][2];
            pp[(int64_t)co1 * Kp + n + 1] = acc[j][3];
        }
    }
}

// dW[i] = sum_c part[c][i] in chunk order; db[co] = sum over voxels of dy (fixed order)
__global__ void conv3_wgrad_reduce(const float *__restrict__ part, int nchunks, int n,
                                   float *__restrict__ dw) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float s = 0.f;
        for (int c = 0; c < nchunks; ++c) s += part[(int64_t)c * n + i];
        dw[i] = s;
    }
}

// bias gradient: one block per output channel, fixed-order tree over voxels
__global__ void __launch_bounds__(256) bias_grad_kernel(const TView dy, int64_t nv, float *__restrict__ db) {
    __shared__ float sm[256];
    const int co = blockIdx.x;
    float s = 0.f;
    for (int64_t v = threadIdx.x; v < nv; v += 256) s += __bfloat162float(dy.p[v * dy.cs + dy.co + co]);
    sm[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) sm[threadIdx.x] += sm[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) db[co] = sm[0];
}

// W'[ci][tap][co] = W[co][26 - tap][ci]  (input-gradient weights), padded rows
__global__ void flip_weights_kernel(const __nv_bfloat16 *__restrict__ W, int Cout, int Cin, int Kp,
                                    __nv_bfloat16 *__restrict__ Wt, int Kpt) {
    const int total = Cin * Kpt;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const int ci = i / Kpt, k = i % Kpt;
        __nv_bfloat16 v = __float2bfloat16(0.f);
        if (k < 27 * Cout) {
            const int tap = k / Cout, co = k % Cout;
            v = W[(int64_t)co * Kp + (26 - tap) * Cin + ci];
        }
        Wt[i] = v;
    }
}

// dy *= (y > 0)   (ReLU backward through the stored activation)
__global__ void relu_bwd_kernel(TView dy, const TView y, int64_t nv, int C) {
    const int64_t total = nv * C;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t v = i / C;
        const int c = (int)(i % C);
        if (!(__bfloat162float(y.p[v * y.cs + y.co + c]) > 0.f))
            dy.p[v * dy.cs + dy.co + c] = __float2bfloat16(0.f);
    }
}

template <int VW> struct BVec;
template <> struct BVec<2> {
    static __device__ __forceinline__ void ld(const __nv_bfloat16 *p, float (&f)[2]) {
        const float2 t = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(p));
        f[0] = t.x; f[1] = t.y;
    }
    static __device__ __forceinline__ void st(__nv_bfloat16 *p, const float (&f)[2]) {
        *reinterpret_cast<__nv_bfloat162 *>(p) = __floats2bfloat162_rn(f[0], f[1]);
    }
};
template <> struct BVec<8> {
    static __device__ __forceinline__ void ld(const __nv_bfloat16 *p, float (&f)[8]) {
        const uint4 u = *reinterpret_cast<const uint4 *>(p);
        const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            __nv_bfloat162 h;
            memcpy(&h, &w[k], 4);
            const float2 t = __bfloat1622float2(h);
            f[2 * k] = t.x; f[2 * k + 1] = t.y;
        }
    }
    static __device__ __forceinline__ void st(__nv_bfloat16 *p, const float (&f)[8]) {
        uint32_t w[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const __nv_bfloat162 h = __floats2bfloat162_rn(f[2 * k], f[2 * k + 1]);
            memcpy(&w[k], &h, 4);
        }
        *reinterpret_cast<uint4 *>(p) = make_uint4(w[0], w[1], w[2], w[3]);
    }
};

// trilinear prolongation of C channels, VW channels per thread (C, channel
// stride and offset multiples of VW)
template <int VW>
__global__ void prolong_kernel(const TView in, const Vol Vc, TView out, const Vol Vf, int C, float scale,
                               int accumulate) {
    const int G = C / VW;
    const int64_t total = Vf.nvox() * G;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int c = (int)(i % G) * VW;
        const int64_t v = i / G;
        int b, z, y, x;
        vox_coords(Vf, v, b, z, y, x);
        float s[VW];
#pragma unroll
        for (int k = 0; k < VW; ++k) s[k] = 0.f;
        const int cz0 = z >> 1, cy0 = y >> 1, cx0 = x >> 1;
        for (int a = 0; a <= (z & 1); ++a)
            for (int bb = 0; bb <= (y & 1); ++bb)
                for (int d = 0; d <= (x & 1); ++d) {
                    const float w = ((z & 1) ? 0.5f : 1.f) * ((y & 1) ? 0.5f : 1.f) * ((x & 1) ? 0.5f : 1.f);
                    const int64_t vc = (((int64_t)b * Vc.Z + cz0 + a) * Vc.Y + cy0 + bb) * Vc.X + cx0 + d;
                    float f[VW];
                    BVec<VW>::ld(in.p + vc * in.cs + in.co + c, f);
#pragma unroll
                    for (int k = 0; k < VW; ++k) s[k] += w * f[k];
                }
        __nv_bfloat16 *o = out.p + v * out.cs + out.co + c;
        float prev[VW];
        if (accumulate) BVec<VW>::ld(o, prev);
#pragma unroll
        for (int k = 0; k < VW; ++k) s[k] = scale * s[k] + (accumulate ? prev[k] : 0.f);
        BVec<VW>::st(o, s);
    }
}

// full-weighting restriction of C channels, VW channels per thread
template <int VW>
__global__ void restrict_kernel(const TView in, const Vol Vf, TView out, const Vol Vc, int C, float scale) {
    const int G = C / VW;
    const int64_t total = Vc.nvox() * G;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int c = (int)(i % G) * VW;
        const int64_t v = i / G;
        int b, z, y, x;
        vox_coords(Vc, v, b, z, y, x);
        float s[VW];
#pragma unroll
        for (int k = 0; k < VW; ++k) s[k] = 0.f;
#pragma unroll
        for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
            for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
                for (int dx = -1; dx <= 1; ++dx) {
                    const int fz = 2 * z + dz, fy = 2 * y + dy, fx = 2 * x + dx;
                    if (fz < 0 || fz >= Vf.Z || fy < 0 || fy >= Vf.Y || fx < 0 || fx >= Vf.X) continue;
                    const float w = (dz ? 0.5f : 1.f) * (dy ? 0.5f : 1.f) * (dx ? 0.5f : 1.f) * 0.125f;
                    const int64_t vf = (((int64_t)b * Vf.Z + fz) * Vf.Y + fy) * Vf.X + fx;
                    float f[VW];
                    BVec<VW>::ld(in.p + vf * in.cs + in.co + c, f);
#pragma unroll
                    for (int k = 0; k < VW; ++k) s[k] += w * f[k];
                }
#pragma unroll
        for (int k = 0; k < VW; ++k) s[k] *= scale;
        BVec<VW>::st(out.p + v * out.cs + out.co + c, s);
    }
}

__global__ void __launch_bounds__(256) mse_kernel(const TView out, const float *__restrict__ target,
                                                  int64_t nv, int Cout, TView grad, float *__restrict__ partial) {
    __shared__ float sm[256];
    float s = 0.f;
    for (int64_t v = (int64_t)blockIdx.x * 256 + threadIdx.x; v < nv; v += (int64_t)gridDim.x * 256) {
        const float d = __bfloat162float(out.p[v * out.cs + out.co]) - target[v];
        s += d * d;
        grad.p[v * grad.cs + grad.co] = __float2bfloat16(2.f * d / (float)nv);
        for (int c = 1; c < Cout; ++c) grad.p[v * grad.cs + grad.co + c] = __float2bfloat16(0.f);
    }
    sm[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) sm[threadIdx.x] += sm[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = sm[0];
}

// Adam on FP32 master parameters, refreshing the BF16 copies (padded rows kept 0).
__global__ void adam_kernel(float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m,
                            float *__restrict__ v, int n, float lr, float b1, float b2, float eps,
                            float bc1, float bc2, __nv_bfloat16 *__restrict__ wb) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
        w[i] = wi;
        if (wb) wb[i] = __float2bfloat16(wi);
    }
}

__global__ void f32_to_bf16_kernel(const float *__restrict__ a, __nv_bfloat16 *__restrict__ b, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = __float2bfloat16(a[i]);
}

// ---- coupling with the FE vectors (native layout, Q1 vertex grid) ----------
// Fine grid = the DOF grid (NI, NJ, NK) of a Q1 operator; coarse grid =
// ((NI+1)/2, (NJ+1)/2, (NK+1)/2), vertex-centred.

// rc[v] = (R r)[v]  (FP32 coarse volume, one batch element)
template <typename T>
__global__ void fe_restrict_kernel(const Grid g, const T *__restrict__ r, float *__restrict__ rc, const Vol Vc) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < Vc.nvox(); i += (int64_t)gridDim.x * blockDim.x) {
        int b, z, y, x;
        vox_coords(Vc, i, b, z, y, x);
        double s = 0.0;
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    const int K = 2 * z + dz, J = 2 * y + dy, I = 2 * x + dx;
                    if (K < 0 || K >= g.NK || J < 0 || J >= g.NJ || I < 0 || I >= g.NI) continue;
                    const double w = (dz ? 0.5 : 1.0) * (dy ? 0.5 : 1.0) * (dx ? 0.5 : 1.0) * 0.125;
                    s += w * (double)r[g.dof(I, J, K)];
                }
        rc[i] = (float)s;
    }
}

// out[0] = sqrt(mean(v^2)) over n values (single block of 1024, fixed order)
__global__ void __launch_bounds__(1024) rms_kernel(const float *__restrict__ v, int64_t n, double *__restrict__ out) {
    __shared__ double sm[1024];
    double s = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += 1024) s += (double)v[i] * (double)v[i];
    sm[threadIdx.x] = s;
    __syncthreads();
    for (int w = 512; w > 0; w >>= 1) {
        if (threadIdx.x < w) sm[threadIdx.x] += sm[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = sqrt(sm[0] / (double)(n > 0 ? n : 1));
}

// network input: channel 0 = rc / scale, channel 1 = lk (coarse log kappa)
__global__ void pack_input_kernel(const float *__restrict__ rc, const float *__restrict__ lk, int64_t n,
                                  const double *__restrict__ scale, TView x0) {
    const double s = scale[0] > 0.0 ? scale[0] : 1.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        *reinterpret_cast<__nv_bfloat162 *>(x0.p + i * x0.cs + x0.co) =
            __floats2bfloat162_rn((float)(rc[i] / s), lk ? lk[i] : 0.f);
}

// FP32 training input [n][2] = (rc / scale, lk)
__global__ void pack_input_f32_kernel(const float *__restrict__ rc, const float *__restrict__ lk, int64_t n,
                                      const double *__restrict__ scale, float *__restrict__ out) {
    const double s = scale[0] > 0.0 ? scale[0] : 1.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        out[2 * i] = (float)(rc[i] / s);
        out[2 * i + 1] = lk ? lk[i] : 0.f;
    }
}

// z (native, T) (+)= scale * P(out channel 0); zero on essential DOFs and pads
template <typename T>
__global__ void fe_prolong_kernel(const Grid g, const TView in, const Vol Vc, T *__restrict__ z,
                                  const double *__restrict__ scale, int accumulate) {
    const double sc = scale ? scale[0] : 1.0;
    const int64_t n = (int64_t)g.NIp * g.NJ * g.NK;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int I = (int)(i % g.NIp);
        const int64_t row = i / g.NIp;
        const int J = (int)(row % g.NJ), K = (int)(row / g.NJ);
        double s = 0.0;
        if (I < g.NI && !g.is_ess(I, J, K)) {
            for (int a = 0; a <= (K & 1); ++a)
                for (int bb = 0; bb <= (J & 1); ++bb)
                    for (int d = 0; d <= (I & 1); ++d) {
                        const double w = ((K & 1) ? 0.5 : 1.0) * ((J & 1) ? 0.5 : 1.0) * ((I & 1) ? 0.5 : 1.0);
                        const int64_t vc = ((int64_t)((K >> 1) + a) * Vc.Y + (J >> 1) + bb) * Vc.X + (I >> 1) + d;
                        s += w * (double)__bfloat162float(in.p[vc * in.cs + in.co]);
                    }
            s *= sc;
        }
        z[i] = accumulate ? (T)((double)z[i] + s) : (T)s;
    }
}

// single-channel FP32 vertex-centred transfers between coarse levels
__global__ void restrict_f32_kernel(const float *__restrict__ f, const Vol Vf, float *__restrict__ c,
                                    const Vol Vc, float scale) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < Vc.nvox(); i += (int64_t)gridDim.x * blockDim.x) {
        int b, z, y, x;
        vox_coords(Vc, i, b, z, y, x);
        float s = 0.f;
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    const int fz = 2 * z + dz, fy = 2 * y + dy, fx = 2 * x + dx;
                    if (fz < 0 || fz >= Vf.Z || fy < 0 || fy >= Vf.Y || fx < 0 || fx >= Vf.X) continue;
                    const float w = (dz ? 0.5f : 1.f) * (dy ? 0.5f : 1.f) * (dx ? 0.5f : 1.f) * 0.125f;
                    s += w * f[(((int64_t)b * Vf.Z + fz) * Vf.Y + fy) * Vf.X + fx];
                }
        c[i] = scale * s;
    }
}
__global__ void prolong_f32_kernel(const float *__restrict__ c, const Vol Vc, float *__restrict__ f,
                                   const Vol Vf) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < Vf.nvox(); i += (int64_t)gridDim.x * blockDim.x) {
        int b, z, y, x;
        vox_coords(Vf, i, b, z, y, x);
        float s = 0.f;
        for (int a = 0; a <= (z & 1); ++a)
            for (int bb = 0; bb <= (y & 1); ++bb)
                for (int d = 0; d <= (x & 1); ++d) {
                    const float w = ((z & 1) ? 0.5f : 1.f) * ((y & 1) ? 0.5f : 1.f) * ((x & 1) ? 0.5f : 1.f);
                    s += w * c[(((int64_t)b * Vc.Z + (z >> 1) + a) * Vc.Y + (y >> 1) + bb) * Vc.X + (x >> 1) + d];
                }
        f[i] = s;
    }
}

// z (native, T) (+)= scale[0] * mult * P(cf) for an FP32 field cf on the
// first coarse level; zero on essential DOFs and pads.  Grid: x over pairs of
// DOFs along a row (2m, 2m+1), y = J, z = K, so a thread does no index
// division and every DOF of the vector has its own thread (a grid-stride loop
// over 17M DOFs left each thread ~115 dependent iterations: 135 us instead of
// the ~25 us its bytes take).
template <typename T>
__global__ void __launch_bounds__(256) fe_prolong_f32_kernel(const Grid g, const float *__restrict__ cf,
                                                             const Vol Vc, T *__restrict__ z,
                                                             const double *__restrict__ scale, double mult,
                                                             int accumulate) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    const int J = blockIdx.y, K = blockIdx.z;
    if (2 * m >= g.NIp) return;
    const double sc = (scale ? scale[0] : 1.0) * mult;
    const int64_t row = ((int64_t)K * g.NJ + J) * g.NIp;
    const int64_t crow = ((int64_t)(K >> 1) * Vc.Y + (J >> 1)) * Vc.X;
    const int oz = (K & 1) ? Vc.Y * Vc.X : 0, oy = (J & 1) ? Vc.X : 0;
    const double wz = (K & 1) ? 0.5 : 1.0, wy = (J & 1) ? 0.5 : 1.0;
    const double ay = oy ? wy : 0.0, az = oz ? wz : 0.0;
    const bool ess_jk = ((g.ess & 1) && K == 0) || ((g.ess & 2) && K == g.NK - 1) ||
                        ((g.ess & 4) && J == 0) || ((g.ess & 8) && J == g.NJ - 1);
#pragma unroll
    for (int h = 0; h < 2; ++h) {  // NIp is a multiple of 4: both DOFs of the pair exist
        const int I = 2 * m + h;
        double s = 0.0;
        if (I < g.NI && !ess_jk && !(((g.ess & 16) && I == 0) || ((g.ess & 32) && I == g.NI - 1))) {
            const int64_t c0 = crow + (I >> 1);
            const int ox = I & 1;
            const double wx = ox ? 0.5 : 1.0;
            // terms with a zero offset repeat the base value with weight 0 (same sum)
            const double f000 = cf[c0], f001 = cf[c0 + ox], f010 = cf[c0 + oy], f011 = cf[c0 + oy + ox];
            const double f100 = cf[c0 + oz], f101 = cf[c0 + oz + ox], f110 = cf[c0 + oz + oy],
                         f111 = cf[c0 + oz + oy + ox];
            const double ax = ox ? wx : 0.0;
            const double y0 = wx * f000 + ax * f001, y1 = wx * f010 + ax * f011;
            const double y2 = wx * f100 + ax * f101, y3 = wx * f110 + ax * f111;
            const double z0 = wy * y0 + ay * y1, z1 = wy * y2 + ay * y3;
            s = sc * (wz * z0 + az * z1);
        }
        T *zp = z + row + I;
        *zp = accumulate ? (T)((double)*zp + s) : (T)s;
    }
}

// energy-loss gradient into the output-gradient buffer:
// dout[v][0] = coef / scale[0] * g[v], other channels 0
__global__ void energy_grad_kernel(const float *__restrict__ gc, int64_t nv, float coef,
                                   const double *__restrict__ scale, TView dout) {
    const float f = (float)(coef / (scale[0] > 0.0 ? scale[0] : 1.0));
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += (int64_t)gridDim.x * blockDim.x) {
        __nv_bfloat16 *o = dout.p + i * dout.cs + dout.co;
        o[0] = __float2bfloat16(f * gc[i]);
        for (int c = 1; c < dout.cs; ++c) o[c] = __float2bfloat16(0.f);
    }
}

// training pair from a PCG iterate: target = (x* - x_k) injected at the
// network vertices (every stride-th DOF), / scale
__global__ void pair_target_kernel(const Grid g, const double *__restrict__ xs, const double *__restrict__ xk,
                                   const Vol Vc, int stride, const double *__restrict__ scale, float *__restrict__ t) {
    const double s = scale[0] > 0.0 ? scale[0] : 1.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < Vc.nvox(); i += (int64_t)gridDim.x * blockDim.x) {
        int b, z, y, x;
        vox_coords(Vc, i, b, z, y, x);
        const int64_t d = g.dof(stride * x, stride * y, stride * z);
        t[i] = (float)((xs[d] - xk[d]) / s);
    }
}

// float input volume [n][2] -> BF16 x0; float channel 0 of the output -> dst
__global__ void f32x2_to_x0_kernel(const float *__restrict__ in, int64_t nv, TView x0) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += (int64_t)gridDim.x * blockDim.x)
        *reinterpret_cast<__nv_bfloat162 *>(x0.p + i * x0.cs + x0.co) = __floats2bfloat162_rn(in[2 * i], in[2 * i + 1]);
}
__global__ void out0_to_f32_kernel(const TView out, int64_t nv, float *__restrict__ dst) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = __bfloat162float(out.p[i * out.cs + out.co]);
}

}  // namespace fg
