// The context behind the opaque ilg_ctx handle.
#pragma once

#include <cstdio>

#include "build.cuh"
#include "ilg.h"
#include "trace_api.cuh"

struct ilg_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    char err[512] = {0};

    // mesh as uploaded
    ilg::DevBuf<float> pos;
    ilg::DevBuf<uint32_t> idx, mat;
    uint32_t n_verts = 0, n_tris = 0;
    bool has_mat = false;
    float max_abs = 0.f;

    // built scene
    ilg::BuildBuffers bb;
    bool built = false;
    ilg_stats stats = {};

    // staging for host-pointer queries
    ilg::DevBuf<float4> ro, rd;
    ilg::DevBuf<int32_t> hprim;
    ilg::DevBuf<float> ht, hu, hv;
    ilg::DevBuf<uint8_t> hocc;

    // device error word: bit 0 = traversal stack exceeded, bit 1 = index out of range, bit 2 = node visit budget
    ilg::DevBuf<uint32_t> derr;
    ilg::DevBuf<unsigned long long> dstats;

    ilg::SceneView view() const
    {
        return ilg::SceneView{bb.nodes, bb.tris, bb.prim_of, stats.n_nodes, stats.n_tris};
    }

    int check_device_error()
    {
        uint32_t h = 0;
        if (cudaMemcpy(&h, derr.ptr, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess) {
            snprintf(err, sizeof(err), "reading the device error word failed");
            return ILG_ECUDA;
        }
        if (h) {
            cudaMemset(derr.ptr, 0, sizeof(uint32_t));
            snprintf(err, sizeof(err), "device reported error flags 0x%x (bit0: traversal stack bound, bit1: node/triangle index out of range, bit2: node visit budget)", h);
            return ILG_EOVERFLOW;
        }
        return ILG_OK;
    }

    void release_all()
    {
        pos.release(); idx.release(); mat.release();
        bb.release_all();
        ro.release(); rd.release(); hprim.release(); ht.release(); hu.release(); hv.release(); hocc.release();
        derr.release(); dstats.release();
    }
};
