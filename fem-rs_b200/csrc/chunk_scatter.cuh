// chunk_scatter.cuh -- device side of the chunked deterministic scatter of the
// unstructured operators (plan: chunk_plan.h).  A CTA holds its chunk's element
// results in shared memory as ys[i * CE + e_local]; per DOF of the chunk's list
// its slots are summed in the listed order and the DOF (owned) or its partial
// (shared) is stored; chunk_shared_kernel adds each shared DOF's
// partials in chunk order.  chunk_stage_lists stages a chunk's lists in shared
// memory and chunk_sums does the sums.  On essential DOFs of a constrained call the
// identity row: y_d (+)= x_d (apply) or 1 (diagonal).
#pragma once
#include <cstdint>

namespace fg {

struct ChunkLists {
    const int32_t *cu_off;     // [n_chunks + 1] start of each chunk's DOF list
    const int32_t *cu_dof;     // [U] global DOF
    const int32_t *cu_pid;     // [U] partial slot of a shared DOF, -1 for a DOF owned by the chunk
    const int32_t *cu_soff;    // [U + 1] start of each DOF's local slots
    const uint16_t *cu_slots;  // local slots i * CE + e_local, increasing per DOF
    void *part;                // [n_part] partial sums of shared DOFs (the apply's precision)
    const int32_t *sh_dof;     // [n_shared] DOFs not owned by one chunk (incl. DOFs of no element)
    const int32_t *sh_off;     // [n_shared + 1] their partial ranges (in chunk order)
    int64_t n_shared;
    int max_nu;                // longest chunk DOF list
};

// Bytes of shared memory a chunk's lists are staged in.
__host__ __device__ inline size_t chunk_list_smem(int nl, int CE, int max_nu) {
    return (sizeof(int32_t) * (3 * (size_t)max_nu + 1) + sizeof(uint16_t) * (size_t)nl * CE + 15) & ~(size_t)15;
}

// Chunk c's lists staged in shared memory (chunk_list_smem bytes).
struct ChunkStage {
    int32_t *sdof, *spid, *soff;  // [MU], [MU], [MU + 1]
    uint16_t *sslot;
    int nu;
};

__device__ __forceinline__ ChunkStage chunk_stage_at(const ChunkLists &L, unsigned char *stage) {
    const int MU = L.max_nu;
    ChunkStage S;
    S.sdof = reinterpret_cast<int32_t *>(stage);
    S.spid = S.sdof + MU;
    S.soff = S.spid + MU;
    S.sslot = reinterpret_cast<uint16_t *>(S.soff + MU + 1);
    S.nu = 0;
    return S;
}

// Block-wide (BT threads): load chunk c's lists into the stage.  No barrier:
// the caller places one before chunk_sums.
template <int BT>
__device__ __forceinline__ void chunk_stage_lists(const ChunkLists &L, int c, ChunkStage &S) {
    const int u0 = __ldg(L.cu_off + c), nu = __ldg(L.cu_off + c + 1) - u0;
    const int s0 = __ldg(L.cu_soff + u0), ns = __ldg(L.cu_soff + u0 + nu) - s0;
    for (int k = threadIdx.x; k < nu; k += BT) {
        S.sdof[k] = __ldg(L.cu_dof + u0 + k);
        S.spid[k] = __ldg(L.cu_pid + u0 + k);
        S.soff[k] = __ldg(L.cu_soff + u0 + k) - s0;
    }
    if (threadIdx.x == 0) S.soff[nu] = ns;
    for (int j = threadIdx.x; j < ns; j += BT) S.sslot[j] = __ldg(L.cu_slots + s0 + j);
    S.nu = nu;
}

// Block-wide (BT threads), after a barrier that follows both the element
// phase (ys complete) and chunk_stage_lists: per DOF of the chunk the sum of
// its slots in the listed order, stored (owned) or as the partial (shared).
template <typename T, int BT>
__device__ __forceinline__ void chunk_sums(const ChunkLists &L, const ChunkStage &S, const T *ys,
                                           const uint8_t *ess, const T *x, T *y, int accumulate, int constrained,
                                           int diag) {
    T *part = reinterpret_cast<T *>(L.part);
    for (int k = threadIdx.x; k < S.nu; k += BT) {
        T s = T(0);
        for (int j = S.soff[k]; j < S.soff[k + 1]; ++j) s += ys[S.sslot[j]];
        const int32_t pid = S.spid[k];
        if (pid >= 0) {
            part[pid] = s;
        } else {
            const int32_t d = S.sdof[k];
            if (constrained && ess && ess[d]) s = diag ? T(1) : x[d];
            y[d] = accumulate ? y[d] + s : s;
        }
    }
}

// DOFs not owned by a single chunk: the partials of their chunks in chunk order
template <typename T>
__global__ void chunk_shared_kernel(const ChunkLists L, const uint8_t *ess, const T *__restrict__ x,
                                    T *__restrict__ y, int accumulate, int constrained, int diag,
                                    const int *skip) {
    if (skip && *skip) return;
    const T *part = reinterpret_cast<const T *>(L.part);
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < L.n_shared;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int32_t d = L.sh_dof[k];
        T s = T(0);
#pragma unroll 4
        for (int j = L.sh_off[k]; j < L.sh_off[k + 1]; ++j) s += part[j];
        if (constrained && ess && ess[d]) s = diag ? T(1) : x[d];
        y[d] = accumulate ? y[d] + s : s;
    }
}

}  // namespace fg
