// Buffers and entry point of the device BVH build (build.cu).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cuda_runtime.h>

#include "bvh8.cuh"

namespace ilg {

// Grow-only device allocation owned by a context.
template <class T>
struct DevBuf {
    T *ptr = nullptr;
    size_t cap = 0;  // elements
    cudaError_t reserve(size_t n)
    {
        if (n <= cap) return cudaSuccess;
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        cap = 0;
        cudaError_t e = cudaMalloc((void **)&ptr, (n ? n : 1) * sizeof(T));
        if (e == cudaSuccess) cap = n;
        return e;
    }
    void release()
    {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        cap = 0;
    }
};

struct BuildBuffers {
    // scratch (valid only during a build)
    DevBuf<float4> tlo_b, thi_b, nlo_b, nhi_b;
    DevBuf<uint32_t> keys_b, keys_alt_b, vals_b, vals_alt_b, arrivals_b, cb_b, counters_b, err_b;
    DevBuf<int2> child_b, range_b;
    DevBuf<int> parent_int_b, parent_leaf_b, cnt_b;
    DevBuf<float> cost_b, dpc_b;
    DevBuf<uint8_t> dpd_b;
    DevBuf<unsigned char> sort_tmp_b;
    DevBuf<uint64_t> qa_b, qb_b;  // work items, 8 bytes each
    // outputs (the built scene)
    DevBuf<Node8> nodes_b;
    DevBuf<Tri> tris_b;
    DevBuf<uint32_t> prim_of_b;

    float4 *tlo, *thi, *nlo, *nhi;
    uint32_t *keys, *keys_alt, *vals, *vals_alt, *arrivals, *cbounds, *counters, *err;
    int2 *child, *range;
    int *parent_int, *parent_leaf, *cnt;
    float *cost, *dpc;  // dpc: 8 collapse costs a binary node
    uint8_t *dpd;       // 16 collapse decisions a binary node
    void *sort_tmp;
    void *qa_raw, *qb_raw;  // two 8-byte work-item queues
    Node8 *nodes;
    Tri *tris;
    uint32_t *prim_of;

    cudaError_t reserve(size_t n, size_t sort_bytes, size_t node_cap, size_t queue_cap, cudaStream_t)
    {
        cudaError_t e;
#define ILG_R(b, k) if ((e = b.reserve(k)) != cudaSuccess) return e;
        ILG_R(tlo_b, n) ILG_R(thi_b, n) ILG_R(nlo_b, n) ILG_R(nhi_b, n)
        ILG_R(keys_b, n) ILG_R(keys_alt_b, n) ILG_R(vals_b, n) ILG_R(vals_alt_b, n) ILG_R(arrivals_b, n)
        ILG_R(cb_b, 8) ILG_R(counters_b, 8) ILG_R(err_b, 1)
        ILG_R(child_b, n) ILG_R(range_b, n) ILG_R(parent_int_b, n) ILG_R(parent_leaf_b, n) ILG_R(cnt_b, n)
        ILG_R(cost_b, n) ILG_R(dpc_b, 8 * n) ILG_R(dpd_b, 16 * n)
        ILG_R(sort_tmp_b, sort_bytes) ILG_R(qa_b, queue_cap) ILG_R(qb_b, queue_cap)
        ILG_R(nodes_b, node_cap) ILG_R(tris_b, n) ILG_R(prim_of_b, n)
#undef ILG_R
        tlo = tlo_b.ptr; thi = thi_b.ptr; nlo = nlo_b.ptr; nhi = nhi_b.ptr;
        keys = keys_b.ptr; keys_alt = keys_alt_b.ptr; vals = vals_b.ptr; vals_alt = vals_alt_b.ptr;
        arrivals = arrivals_b.ptr; cbounds = cb_b.ptr; counters = counters_b.ptr; err = err_b.ptr;
        child = child_b.ptr; range = range_b.ptr; parent_int = parent_int_b.ptr; parent_leaf = parent_leaf_b.ptr;
        cnt = cnt_b.ptr; cost = cost_b.ptr; dpc = dpc_b.ptr; dpd = dpd_b.ptr;
        sort_tmp = sort_tmp_b.ptr; qa_raw = qa_b.ptr; qb_raw = qb_b.ptr;
        nodes = nodes_b.ptr; tris = tris_b.ptr; prim_of = prim_of_b.ptr;
        return cudaSuccess;
    }

    // Frees the scratch, keeps the built scene.
    void release_scratch()
    {
        tlo_b.release(); thi_b.release(); nlo_b.release(); nhi_b.release();
        keys_b.release(); keys_alt_b.release(); vals_b.release(); vals_alt_b.release(); arrivals_b.release();
        child_b.release(); range_b.release(); parent_int_b.release(); parent_leaf_b.release();
        cnt_b.release(); cost_b.release(); dpc_b.release(); dpd_b.release();
        sort_tmp_b.release(); qa_b.release(); qb_b.release();
    }

    void release_all()
    {
        release_scratch();
        cb_b.release(); counters_b.release(); err_b.release();
        nodes_b.release(); tris_b.release(); prim_of_b.release();
    }
};

struct BuildResult {
    float min_step = 0.f;   // in: smallest quantisation step (world units)
    bool treelets = true;   // in: restructure the binary tree by treelets before the collapse
    uint32_t n_nodes = 0;   // out
    uint32_t n_tris = 0;    // out
    uint32_t depth = 0;     // out
};

// Returns 0 on success, else an ilg_status code with `err` filled in.
int bvh_build(BuildBuffers &B, const float *d_pos, uint32_t n_verts, const uint32_t *d_idx, uint32_t n,
              cudaStream_t st, BuildResult &res, char *err, size_t err_len);

}  // namespace ilg
