// unet_host.cuh -- host side of the learned coarse correction (included by
// femgpu.cu, single translation unit).
//
// Network (channels C0, C1, C2; default 16, 32, 48, ~246k parameters), on a
// volume S0 (odd extents) with levels S1 = (S0+1)/2, S2 = (S1+1)/2:
//   level 0: a0 = relu(conv(x; 2->C0)),  h0 = relu(conv(a0; C0->C0))
//   level 1: x1 = R h0,  a1 = relu(conv(x1; C0->C1)),  h1 = relu(conv(a1; C1->C1))
//   level 2: x2 = R h1,  a2 = relu(conv(x2; C1->C2)),  h2 = relu(conv(a2; C2->C2))
//   up 1:    g1 = relu(conv([P h2, h1]; C2+C1->C1))
//   up 0:    g0 = relu(conv([P g1, h0]; C1+C0->C0))
//   out = conv(g0; C0->8), channel 0 is the prediction.
// R = full-weighting restriction, P = trilinear prolongation (fixed).
#pragma once
#include <cuda_bf16.h>

#include <vector>

#include "unet_kernels.cuh"
#include "unet_tc.cuh"

namespace fg {

struct ConvLayer {
    int cin = 0, cout = 0, kp = 0, kpt = 0;  // kp: padded K of W, kpt: padded K of the flipped W
    float *w = nullptr, *b = nullptr;         // FP32 master parameters (w: [cout][kp])
    __nv_bfloat16 *wb = nullptr;               // BF16 copy used by the kernels
    float *gw = nullptr, *gb = nullptr;       // gradients
    float *mw = nullptr, *vw = nullptr, *mb = nullptr, *vb = nullptr;  // Adam moments
};

enum { L0A, L0B, L1A, L1B, L2A, L2B, L1C, L0C, LOUT, NLAYERS };

struct UnetBufs {
    int B = 0, Z = 0, Y = 0, X = 0;
    Vol v0{}, v1{}, v2{};
    std::vector<__nv_bfloat16 *> all;
    __nv_bfloat16 *x0 = nullptr, *a0 = nullptr, *cat0 = nullptr, *x1 = nullptr, *a1 = nullptr,
                  *cat1 = nullptr, *x2 = nullptr, *a2 = nullptr, *h2 = nullptr, *g1 = nullptr,
                  *g0 = nullptr, *out = nullptr;
    // gradients (same shapes)
    __nv_bfloat16 *da0 = nullptr, *dcat0 = nullptr, *dx1 = nullptr, *da1 = nullptr, *dcat1 = nullptr,
                  *dx2 = nullptr, *da2 = nullptr, *dh2 = nullptr, *dg1 = nullptr, *dg0 = nullptr,
                  *dout = nullptr;
    float *target = nullptr, *part = nullptr, *msep = nullptr;
    size_t part_n = 0;
};

}  // namespace fg

struct fg_unet {
    int device = 0;
    int C0 = 16, C1 = 32, C2 = 48;
    fg::ConvLayer L[fg::NLAYERS];
    fg::UnetBufs buf;
    __nv_bfloat16 *wflip = nullptr;
    size_t wflip_n = 0;
    int step = 0;
    cudaStream_t stream = nullptr;
    int tc = 0;            // FG_UNET_TC=1: convolutions on tcgen05 where the shapes allow (default mma.sync)
    int *d_err = nullptr;  // the network's own device error word
    int *err = nullptr;    // error word the convolutions report to (d_err, or the solving operator's)
};

namespace fg {

static inline int kpad(int k) { return (k + 15) / 16 * 16; }

static float hash_uniform(uint64_t i) {  // splitmix64 -> [-1, 1)
    uint64_t z = i + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z = z ^ (z >> 31);
    return (float)((double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0);
}

static int unet_layer_alloc(ConvLayer &l, int cin, int cout, uint64_t seed) {
    l.cin = cin;
    l.cout = cout;
    l.kp = kpad(27 * cin);
    l.kpt = kpad(27 * cout);
    const size_t nw = (size_t)cout * l.kp;
    float **f[] = {&l.w, &l.gw, &l.mw, &l.vw};
    for (float **p : f) {
        CK(cudaMalloc(p, nw * sizeof(float)));
        CK(cudaMemset(*p, 0, nw * sizeof(float)));
    }
    float **fb[] = {&l.b, &l.gb, &l.mb, &l.vb};
    for (float **p : fb) {
        CK(cudaMalloc(p, cout * sizeof(float)));
        CK(cudaMemset(*p, 0, cout * sizeof(float)));
    }
    CK(cudaMalloc(&l.wb, nw * sizeof(__nv_bfloat16)));
    // He-uniform init, deterministic; padded columns stay zero
    std::vector<float> h(nw, 0.f);
    const float a = std::sqrt(6.0f / (27.0f * cin));
    for (int co = 0; co < cout; ++co)
        for (int k = 0; k < 27 * cin; ++k) h[(size_t)co * l.kp + k] = a * hash_uniform(seed * 1000003ull + (uint64_t)co * 100000 + k);
    CK(cudaMemcpy(l.w, h.data(), nw * sizeof(float), cudaMemcpyHostToDevice));
    f32_to_bf16_kernel<<<64, 256>>>(l.w, l.wb, (int64_t)nw);
    CK(cudaGetLastError());
    FG_LEGACY_FENCE();
    return FG_OK;
}

static void unet_free_bufs(UnetBufs &b) {
    for (auto *p : b.all) cudaFree(p);
    b.all.clear();
    if (b.target) cudaFree(b.target);
    if (b.part) cudaFree(b.part);
    if (b.msep) cudaFree(b.msep);
    b = UnetBufs{};
}

static int unet_ensure_bufs(fg_unet *u, int B, int Z, int Y, int X) {
    UnetBufs &b = u->buf;
    if (b.B == B && b.Z == Z && b.Y == Y && b.X == X) return FG_OK;
    unet_free_bufs(b);
    // every level must have odd extents (vertex-centred transfers): Z, Y, X = 1 mod 4
    if (Z % 4 != 1 || Y % 4 != 1 || X % 4 != 1 || Z < 5 || Y < 5 || X < 5)
        return fail(FG_UNSUPPORTED, "network volume extents must be 1 mod 4 and >= 5 (got %d %d %d)", Z, Y, X);
    b.B = B; b.Z = Z; b.Y = Y; b.X = X;
    b.v0 = Vol{B, Z, Y, X};
    b.v1 = Vol{B, (Z + 1) / 2, (Y + 1) / 2, (X + 1) / 2};
    b.v2 = Vol{B, (b.v1.Z + 1) / 2, (b.v1.Y + 1) / 2, (b.v1.X + 1) / 2};
    const int C0 = u->C0, C1 = u->C1, C2 = u->C2;
    auto mk = [&](__nv_bfloat16 **p, const Vol &v, int c) -> int {
        const size_t n = (size_t)v.nvox() * c;
        CK(cudaMalloc(p, n * sizeof(__nv_bfloat16)));
        CK(cudaMemset(*p, 0, n * sizeof(__nv_bfloat16)));
        FG_LEGACY_FENCE();
        b.all.push_back(*p);
        return FG_OK;
    };
    int rc;
    if ((rc = mk(&b.x0, b.v0, 2)) || (rc = mk(&b.a0, b.v0, C0)) || (rc = mk(&b.cat0, b.v0, C1 + C0)) ||
        (rc = mk(&b.x1, b.v1, C0)) || (rc = mk(&b.a1, b.v1, C1)) || (rc = mk(&b.cat1, b.v1, C2 + C1)) ||
        (rc = mk(&b.x2, b.v2, C1)) || (rc = mk(&b.a2, b.v2, C2)) || (rc = mk(&b.h2, b.v2, C2)) ||
        (rc = mk(&b.g1, b.v1, C1)) || (rc = mk(&b.g0, b.v0, C0)) || (rc = mk(&b.out, b.v0, 8)) ||
        (rc = mk(&b.da0, b.v0, C0)) || (rc = mk(&b.dcat0, b.v0, C1 + C0)) || (rc = mk(&b.dx1, b.v1, C0)) ||
        (rc = mk(&b.da1, b.v1, C1)) || (rc = mk(&b.dcat1, b.v1, C2 + C1)) || (rc = mk(&b.dx2, b.v2, C1)) ||
        (rc = mk(&b.da2, b.v2, C2)) || (rc = mk(&b.dh2, b.v2, C2)) || (rc = mk(&b.dg1, b.v1, C1)) ||
        (rc = mk(&b.dg0, b.v0, C0)) || (rc = mk(&b.dout, b.v0, 8)))
        return rc;
    CK(cudaMalloc(&b.target, sizeof(float) * b.v0.nvox()));
    CK(cudaMalloc(&b.msep, sizeof(float) * 1024));
    return FG_OK;
}

template <int NT, int KS>
static void conv_launch(fg_unet *u, bool tapmajor, int blocks, const TView &in, const Vol &V,
                        const __nv_bfloat16 *w, int cin, int kp, const float *bias, TView out, int relu) {
    if (tapmajor)
        conv3_fwd16_kernel<NT, KS><<<blocks, 128, 0, u->stream>>>(in, V, cin, w, kp, bias, out, relu);
    else
        conv3_fwd_kernel<NT, KS><<<blocks, 128, 0, u->stream>>>(in, V, cin, w, kp, bias, out, relu);
}

template <int KS>
static int conv_fwd_ks(fg_unet *u, const TView &in, const Vol &V, const __nv_bfloat16 *w, int cin, int cout,
                       int kp, const float *bias, TView out, int relu) {
    const int64_t tiles = (V.nvox() + 15) / 16;
    const int blocks = (int)((tiles + (4 / KS) - 1) / (4 / KS));
    const bool tm = cin % 16 == 0 && in.cs % 4 == 0 && in.co % 4 == 0;
    switch (cout / 8) {
    case 1: conv_launch<1, KS>(u, tm, blocks, in, V, w, cin, kp, bias, out, relu); break;
    case 2: conv_launch<2, KS>(u, tm, blocks, in, V, w, cin, kp, bias, out, relu); break;
    case 4: conv_launch<4, KS>(u, tm, blocks, in, V, w, cin, kp, bias, out, relu); break;
    case 6: conv_launch<6, KS>(u, tm, blocks, in, V, w, cin, kp, bias, out, relu); break;
    case 8: conv_launch<8, KS>(u, tm, blocks, in, V, w, cin, kp, bias, out, relu); break;
    case 10: conv_launch<10, KS>(u, tm, blocks, in, V, w, cin, kp, bias, out, relu); break;
    default: return fail(FG_UNSUPPORTED, "conv output channels %d not supported", cout);
    }
    CK(cudaGetLastError());
    return FG_OK;
}

template <int NPAD>
static void conv_tc_launch(fg_unet *u, const TView &in, const Vol &V, const __nv_bfloat16 *w, int cin, int cinp,
                           int kp, int cout, const float *bias, TView out, int relu) {
    const int blocks = (int)((V.nvox() + 127) / 128);
    int G, S;
    conv_tc_plan(NPAD, cinp, blocks, G, S);
    conv3_fwd_tc_kernel<NPAD><<<blocks, 128, conv_tc_smem_bytes(NPAD, cinp, G, S), u->stream>>>(
        in, V, cin, cinp, w, kp, cout, bias, out, relu, G, S, u->err);
}

// Shapes the tcgen05 convolution takes: channel counts multiples of 8 (the
// 2-channel input layer stays on mma.sync), 16-byte aligned channel views.
static bool conv_tc_ok(const fg_unet *u, const TView &in, const TView &out, int cin, int cout, int kp) {
    return u->tc && cin % 8 == 0 && cout % 8 == 0 && cout <= 64 && (cin + 15) / 16 * 16 <= TC_MAX_CINP &&
           in.cs % 8 == 0 && in.co % 8 == 0 && out.cs % 8 == 0 && out.co % 8 == 0 && kp % 16 == 0;
}

// Every tcgen05 convolution instance may use up to TC_SMEM_MAX bytes of
// dynamic shared memory (set once per network, outside any stream capture).
static int conv_tc_init() {
    CK(cudaFuncSetAttribute(conv3_fwd_tc_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM_MAX));
    CK(cudaFuncSetAttribute(conv3_fwd_tc_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM_MAX));
    CK(cudaFuncSetAttribute(conv3_fwd_tc_kernel<48>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM_MAX));
    CK(cudaFuncSetAttribute(conv3_fwd_tc_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM_MAX));
    return FG_OK;
}

// mma.sync with the K split chosen so that about 148 x 32 warps are in
// flight; tcgen05 instead where the network asks for it and the shapes allow
// (on the B200 the mma.sync kernels measured faster at every volume from 9^3
// to 2 x 65^3, forward and backward)
static int conv_fwd(fg_unet *u, const ConvLayer &l, const TView &in, const Vol &V, const __nv_bfloat16 *w,
                    int cin, int cout, int kp, const float *bias, TView out, int relu) {
    (void)l;
    if (conv_tc_ok(u, in, out, cin, cout, kp)) {
        const int cinp = (cin + 15) / 16 * 16;
        switch ((cout + 15) / 16) {
        case 1: conv_tc_launch<16>(u, in, V, w, cin, cinp, kp, cout, bias, out, relu); break;
        case 2: conv_tc_launch<32>(u, in, V, w, cin, cinp, kp, cout, bias, out, relu); break;
        case 3: conv_tc_launch<48>(u, in, V, w, cin, cinp, kp, cout, bias, out, relu); break;
        default: conv_tc_launch<64>(u, in, V, w, cin, cinp, kp, cout, bias, out, relu); break;
        }
        CK(cudaGetLastError());
        return FG_OK;
    }
    const int64_t tiles = (V.nvox() + 15) / 16;
    if (tiles >= 148 * 32) return conv_fwd_ks<1>(u, in, V, w, cin, cout, kp, bias, out, relu);
    if (tiles >= 148 * 16) return conv_fwd_ks<2>(u, in, V, w, cin, cout, kp, bias, out, relu);
    return conv_fwd_ks<4>(u, in, V, w, cin, cout, kp, bias, out, relu);
}

static int layer_fwd(fg_unet *u, int li, const TView &in, const Vol &V, TView out, int relu) {
    const ConvLayer &l = u->L[li];
    return conv_fwd(u, l, in, V, l.wb, l.cin, l.cout, l.kp, l.b, out, relu);
}

static void grid_launch(int64_t n, int &blocks) { blocks = (int)std::min<int64_t>((n + 255) / 256, 148 * 16); }

static bool vec8(const TView &a, const TView &b, int C) {
    return C % 8 == 0 && a.cs % 8 == 0 && a.co % 8 == 0 && b.cs % 8 == 0 && b.co % 8 == 0;
}

// channel-wise trilinear prolongation Vc -> Vf (out = scale P in (+ out))
static void launch_prolong(fg_unet *u, const TView &in, const Vol &Vc, TView out, const Vol &Vf, int C,
                           float scale, int accumulate) {
    int blocks;
    if (vec8(in, out, C)) {
        grid_launch(Vf.nvox() * (C / 8), blocks);
        prolong_kernel<8><<<blocks, 256, 0, u->stream>>>(in, Vc, out, Vf, C, scale, accumulate);
    } else {
        grid_launch(Vf.nvox() * (C / 2), blocks);
        prolong_kernel<2><<<blocks, 256, 0, u->stream>>>(in, Vc, out, Vf, C, scale, accumulate);
    }
}

// channel-wise full-weighting restriction Vf -> Vc (out = scale R in)
static void launch_restrict(fg_unet *u, const TView &in, const Vol &Vf, TView out, const Vol &Vc, int C,
                            float scale) {
    int blocks;
    // 8 channels per thread only when that still gives a few threads per SM lane
    if (vec8(in, out, C) && Vc.nvox() * (C / 8) >= 148 * 512) {
        grid_launch(Vc.nvox() * (C / 8), blocks);
        restrict_kernel<8><<<blocks, 256, 0, u->stream>>>(in, Vf, out, Vc, C, scale);
    } else {
        grid_launch(Vc.nvox() * (C / 2), blocks);
        restrict_kernel<2><<<blocks, 256, 0, u->stream>>>(in, Vf, out, Vc, C, scale);
    }
}

static int unet_forward(fg_unet *u) {
    UnetBufs &b = u->buf;
    const int C0 = u->C0, C1 = u->C1, C2 = u->C2;
    int rc;
    const TView x0{b.x0, 2, 0}, a0{b.a0, C0, 0}, h0{b.cat0, C1 + C0, C1}, x1{b.x1, C0, 0},
        a1{b.a1, C1, 0}, h1{b.cat1, C2 + C1, C2}, x2{b.x2, C1, 0}, a2{b.a2, C2, 0}, h2{b.h2, C2, 0},
        up1{b.cat1, C2 + C1, 0}, cat1{b.cat1, C2 + C1, 0}, g1{b.g1, C1, 0}, up0{b.cat0, C1 + C0, 0},
        cat0{b.cat0, C1 + C0, 0}, g0{b.g0, C0, 0}, out{b.out, 8, 0};
    if ((rc = layer_fwd(u, L0A, x0, b.v0, a0, 1)) || (rc = layer_fwd(u, L0B, a0, b.v0, h0, 1))) return rc;
    launch_restrict(u, h0, b.v0, x1, b.v1, C0, 1.f);
    if ((rc = layer_fwd(u, L1A, x1, b.v1, a1, 1)) || (rc = layer_fwd(u, L1B, a1, b.v1, h1, 1))) return rc;
    launch_restrict(u, h1, b.v1, x2, b.v2, C1, 1.f);
    if ((rc = layer_fwd(u, L2A, x2, b.v2, a2, 1)) || (rc = layer_fwd(u, L2B, a2, b.v2, h2, 1))) return rc;
    launch_prolong(u, h2, b.v2, up1, b.v1, C2, 1.f, 0);
    if ((rc = layer_fwd(u, L1C, cat1, b.v1, g1, 1))) return rc;
    launch_prolong(u, g1, b.v1, up0, b.v0, C1, 1.f, 0);
    if ((rc = layer_fwd(u, L0C, cat0, b.v0, g0, 1)) || (rc = layer_fwd(u, LOUT, g0, b.v0, out, 0))) return rc;
    CK(cudaGetLastError());
    return FG_OK;
}

// gradient of one layer: weights/bias from (in, dy); optional input gradient din
static int layer_bwd(fg_unet *u, int li, const TView &in, const Vol &V, const TView &dy, TView *din) {
    ConvLayer &l = u->L[li];
    UnetBufs &b = u->buf;
    const int64_t nv = V.nvox();
    const int chunk = 4096;
    const int nchunks = (int)((nv + chunk - 1) / chunk);
    const size_t need = (size_t)nchunks * l.cout * l.kp;
    if (need > b.part_n) {
        if (b.part) cudaFree(b.part);
        CK(cudaMalloc(&b.part, need * sizeof(float)));
        b.part_n = need;
    }
    dim3 g((l.kp + 31) / 32, nchunks);
    conv3_wgrad_kernel<<<g, 128, 0, u->stream>>>(in, V, l.cin, dy, l.cout, l.kp, chunk, b.part);
    conv3_wgrad_reduce<<<64, 256, 0, u->stream>>>(b.part, nchunks, l.cout * l.kp, l.gw);
    bias_grad_kernel<<<l.cout, 256, 0, u->stream>>>(dy, nv, l.gb);
    CK(cudaGetLastError());
    if (din) {
        const size_t nf = (size_t)l.cin * l.kpt;
        if (nf > u->wflip_n) {
            if (u->wflip) cudaFree(u->wflip);
            CK(cudaMalloc(&u->wflip, nf * sizeof(__nv_bfloat16)));
            u->wflip_n = nf;
        }
        flip_weights_kernel<<<64, 256, 0, u->stream>>>(l.wb, l.cout, l.cin, l.kp, u->wflip, l.kpt);
        int rc = conv_fwd(u, l, dy, V, u->wflip, l.cout, l.cin, l.kpt, nullptr, *din, 0);
        if (rc) return rc;
    }
    return FG_OK;
}

static int relu_bwd(fg_unet *u, TView dy, const TView &y, const Vol &V, int C) {
    int blocks;
    grid_launch(V.nvox() * C, blocks);
    relu_bwd_kernel<<<blocks, 256, 0, u->stream>>>(dy, y, V.nvox(), C);
    CK(cudaGetLastError());
    return FG_OK;
}

// Backward pass from d(out) (already in buf.dout); fills every layer's gw/gb.
static int unet_backward(fg_unet *u) {
    UnetBufs &b = u->buf;
    const int C0 = u->C0, C1 = u->C1, C2 = u->C2;
    int rc;
    const TView x0{b.x0, 2, 0}, a0{b.a0, C0, 0}, h0{b.cat0, C1 + C0, C1}, x1{b.x1, C0, 0},
        a1{b.a1, C1, 0}, h1{b.cat1, C2 + C1, C2}, x2{b.x2, C1, 0}, a2{b.a2, C2, 0}, h2{b.h2, C2, 0},
        cat1{b.cat1, C2 + C1, 0}, g1{b.g1, C1, 0}, cat0{b.cat0, C1 + C0, 0}, g0{b.g0, C0, 0};
    TView dout{b.dout, 8, 0}, dg0{b.dg0, C0, 0}, dcat0{b.dcat0, C1 + C0, 0}, dup0{b.dcat0, C1 + C0, 0},
        dh0{b.dcat0, C1 + C0, C1}, dg1{b.dg1, C1, 0}, dcat1{b.dcat1, C2 + C1, 0}, dup1{b.dcat1, C2 + C1, 0},
        dh1{b.dcat1, C2 + C1, C2}, dh2{b.dh2, C2, 0}, da2{b.da2, C2, 0}, dx2{b.dx2, C1, 0},
        da1{b.da1, C1, 0}, dx1{b.dx1, C0, 0}, da0{b.da0, C0, 0};
    if ((rc = layer_bwd(u, LOUT, g0, b.v0, dout, &dg0))) return rc;
    if ((rc = relu_bwd(u, dg0, g0, b.v0, C0))) return rc;
    if ((rc = layer_bwd(u, L0C, cat0, b.v0, dg0, &dcat0))) return rc;
    // P^T = 8 R : gradient of the level-1 output g1 from the prolongated channels
    launch_restrict(u, dup0, b.v0, dg1, b.v1, C1, 8.f);
    if ((rc = relu_bwd(u, dg1, g1, b.v1, C1))) return rc;
    if ((rc = layer_bwd(u, L1C, cat1, b.v1, dg1, &dcat1))) return rc;
    launch_restrict(u, dup1, b.v1, dh2, b.v2, C2, 8.f);
    if ((rc = relu_bwd(u, dh2, h2, b.v2, C2))) return rc;
    if ((rc = layer_bwd(u, L2B, a2, b.v2, dh2, &da2))) return rc;
    if ((rc = relu_bwd(u, da2, a2, b.v2, C2))) return rc;
    if ((rc = layer_bwd(u, L2A, x2, b.v2, da2, &dx2))) return rc;
    // R^T = P / 8 : add the down-path gradient to the skip gradient of h1
    launch_prolong(u, dx2, b.v2, dh1, b.v1, C1, 0.125f, 1);
    if ((rc = relu_bwd(u, dh1, h1, b.v1, C1))) return rc;
    if ((rc = layer_bwd(u, L1B, a1, b.v1, dh1, &da1))) return rc;
    if ((rc = relu_bwd(u, da1, a1, b.v1, C1))) return rc;
    if ((rc = layer_bwd(u, L1A, x1, b.v1, da1, &dx1))) return rc;
    launch_prolong(u, dx1, b.v1, dh0, b.v0, C0, 0.125f, 1);
    if ((rc = relu_bwd(u, dh0, h0, b.v0, C0))) return rc;
    if ((rc = layer_bwd(u, L0B, a0, b.v0, dh0, &da0))) return rc;
    if ((rc = relu_bwd(u, da0, a0, b.v0, C0))) return rc;
    if ((rc = layer_bwd(u, L0A, x0, b.v0, da0, nullptr))) return rc;
    CK(cudaGetLastError());
    return FG_OK;
}

}  // namespace fg
