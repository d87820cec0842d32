// chunk_plan.h -- host-side plan of the chunked deterministic scatter shared
// by the unstructured operators (tetrahedra, Hex8).
//
// The elements are put in a Morton order of their centroids and cut into
// chunks of CE consecutive elements, one CTA each.  Per chunk the plan lists
// the DOFs its elements touch (ascending), each with its element-local slots
// i * CE + e_local (ascending), and marks a DOF *owned* by the chunk when all
// of its elements lie in that chunk.  Every other DOF -- touched by several
// chunks, or by none -- gets one partial slot per touching chunk, in chunk
// order; chunk_shared_kernel (chunk_scatter.cuh) adds them in that order.
#pragma once
#include <algorithm>
#include <cstdint>
#include <vector>

namespace fg {

// Morton key of a point in the box [lo, lo + ext): 21 bits per axis, interleaved
inline uint64_t morton_key(const double *p, const double *lo, const double *ext) {
    uint64_t key = 0;
    uint32_t v[3];
    for (int a = 0; a < 3; ++a) {
        double f = ext[a] > 0.0 ? (p[a] - lo[a]) / ext[a] : 0.0;
        f = std::min(std::max(f, 0.0), 1.0);
        v[a] = (uint32_t)std::min<double>(f * 2097152.0, 2097151.0);
    }
    for (int b = 20; b >= 0; --b)
        for (int a = 0; a < 3; ++a) key = (key << 1) | ((v[a] >> b) & 1u);
    return key;
}

// perm[n] = the element at position n of the Morton order of the centroids
// cen[E][3] (stable: ties keep the caller's order)
inline void morton_order(const std::vector<double> &cen, int64_t E, std::vector<int32_t> &perm) {
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int64_t e = 0; e < E; ++e)
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], cen[3 * e + a]);
            hi[a] = std::max(hi[a], cen[3 * e + a]);
        }
    const double ext[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
    std::vector<uint64_t> key(E);
    for (int64_t e = 0; e < E; ++e) key[e] = morton_key(&cen[3 * e], lo, ext);
    perm.resize(E);
    for (int64_t e = 0; e < E; ++e) perm[e] = (int32_t)e;
    std::stable_sort(perm.begin(), perm.end(), [&](int32_t a, int32_t b) { return key[a] < key[b]; });
}

struct ChunkPlan {
    std::vector<int32_t> cu_off, cu_dof, cu_pid, cu_soff, sh_dof, sh_off;
    std::vector<uint16_t> cu_slots;
    int max_nu = 0;
    int64_t n_chunks = 0, n_part = 0;
};

// smap: element map [Es][nl] in chunk order (an entry < 0: padding, no DOF);
// requires nl * CE <= 65536 (16-bit local slots).
inline void plan_chunk_lists(const std::vector<int32_t> &smap, int64_t Es, int64_t N, int nl, int CE,
                             ChunkPlan &P) {
    const int64_t nch = (Es + CE - 1) / CE;
    P.n_chunks = nch;
    P.cu_off.assign(nch + 1, 0);
    P.cu_dof.clear();
    P.cu_soff.clear();
    P.cu_slots.clear();
    P.cu_slots.reserve((size_t)Es * nl);
    P.max_nu = 0;
    std::vector<int32_t> nchk(N, 0);
    std::vector<std::pair<int32_t, int32_t>> pr;
    for (int64_t c = 0; c < nch; ++c) {
        const int64_t e0 = c * CE;
        const int ne = (int)std::min<int64_t>(CE, Es - e0);
        pr.clear();
        for (int el = 0; el < ne; ++el)
            for (int i = 0; i < nl; ++i) {
                const int32_t d = smap[(size_t)(e0 + el) * nl + i];
                if (d >= 0) pr.push_back({d, i * CE + el});
            }
        std::sort(pr.begin(), pr.end());
        int nu = 0;
        for (size_t k = 0; k < pr.size(); ++k) {
            if (k == 0 || pr[k].first != pr[k - 1].first) {
                P.cu_dof.push_back(pr[k].first);
                P.cu_soff.push_back((int32_t)P.cu_slots.size());
                ++nchk[pr[k].first];
                ++nu;
            }
            P.cu_slots.push_back((uint16_t)pr[k].second);
        }
        P.cu_off[c + 1] = P.cu_off[c] + nu;
        P.max_nu = std::max(P.max_nu, nu);
    }
    P.cu_soff.push_back((int32_t)P.cu_slots.size());
    std::vector<int32_t> base(N, -1);
    P.sh_dof.clear();
    P.sh_off.assign(1, 0);
    for (int64_t d = 0; d < N; ++d)
        if (nchk[d] != 1) {
            base[d] = P.sh_off.back();
            P.sh_dof.push_back((int32_t)d);
            P.sh_off.push_back(P.sh_off.back() + nchk[d]);
        }
    P.n_part = P.sh_off.back();
    P.cu_pid.resize(P.cu_dof.size());
    for (size_t u = 0; u < P.cu_dof.size(); ++u) {  // chunks in order, so partials land in chunk order
        const int32_t d = P.cu_dof[u];
        P.cu_pid[u] = nchk[d] == 1 ? -1 : base[d]++;
    }
}

}  // namespace fg
