// The context behind the opaque ilg_ctx handle.
#pragma once

#include <cstdio>
#include <cstring>
#include <vector>

#include "build.cuh"
#include "ilg.h"
#include "trace_api.cuh"
#include "render.cuh"
#include "mlp.cuh"
#include "postproc.cuh"

namespace ilg {
class HostPool;  // hostpool.h
// noalloc.cu: the device address of the allocation-free query's fixed array
// on the current device, with the traversal kernel it launches loaded.
cudaError_t noalloc_prepare(void **out);
}  // namespace ilg

struct ilg_ctx {
    int device = 0;
    uint32_t build_flags = 0;  // ILG_BUILD_*
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // two more streams for chunked host-buffer queries (made on first use)
    cudaStream_t side[2] = {nullptr, nullptr};
    cudaEvent_t side_ev[3] = {nullptr, nullptr, nullptr};
    char err[512] = {0};
    // device address of the fixed array ilg_intersect_noalloc stages through
    // (looked up by ilg_create; null if that failed)
    void *noalloc_scratch = nullptr;

    // mesh as uploaded
    ilg::DevBuf<float> pos;
    ilg::DevBuf<uint32_t> idx, mat;
    uint32_t n_verts = 0, n_tris = 0;
    bool has_mat = false;
    float max_abs = 0.f;
    float scene_lo[3] = {0.f, 0.f, 0.f}, scene_hi[3] = {1.f, 1.f, 1.f};

    // built scene
    ilg::BuildBuffers bb;
    bool built = false;
    ilg_stats stats = {};

    // progressive accumulation (AccumulationBuffer) and tone-mapping scratch
    ilg::DevBuf<float> post_acc, post_in, post_out, post_scratch;
    uint32_t post_pixels = 0, post_frames = 0;

    // the watertight test's vertex records (three float4 per triangle record)
    ilg::DevBuf<float4> raw_tris;
    bool raw_ready = false;

    // staging for host-pointer queries
    ilg::DevBuf<float4> ro, rd;
    // three page-locked slots for queries from pageable host memory, and the
    // host threads that copy through them (made on first use)
    void *pin_buf = nullptr;
    cudaEvent_t pin_ev[3] = {nullptr, nullptr, nullptr};
    ilg::HostPool *host_pool = nullptr;
    ilg::DevBuf<int32_t> hprim;
    ilg::DevBuf<float> ht, hu, hv;
    ilg::DevBuf<uint8_t> hocc;

    // device error word: bit 0 = traversal stack exceeded, bit 1 = index out of range, bit 2 = node visit budget
    ilg::DevBuf<uint32_t> derr;
    ilg::DevBuf<unsigned long long> dstats;

    // path tracing: scene attributes
    ilg::DevBuf<ilg::Mat> mats;
    uint32_t n_mats = 0;
    ilg::DevBuf<ilg::Light> lights;
    ilg::DevBuf<uint2> light_range;  // per light: (first triangle, triangle count)
    uint32_t n_lights = 0;
    uint2 light_range_host[ilg::kMaxLights] = {};
    float inf_escape = 0.f;          // number of infinite lights
    bool lights_use_mesh = false;    // some light samples the uploaded mesh's triangles
    uint32_t mesh_gen = 0;           // bumped by every ilg_set_mesh / ilg_load
    uint32_t lights_mesh_gen = 0;    // mesh_gen the mesh lights' areas were computed for
    ilg::DevBuf<uint32_t> tri_attr, light_of_prim;
    bool attr_dirty = true;
    // path tracing: wavefront buffers
    ilg::DevBuf<float4> q_o0, q_d0, q_o1, q_d1, beta, s_o, s_d, s_c, accum, accum_direct, accum_albedo;
    ilg::DevBuf<uint32_t> q_p0, q_p1, counts, path_scene, s_sid;
    ilg::DevBuf<ilg::SceneRec> scene_table;
    ilg::DevBuf<int> hit_tri;
    ilg::DevBuf<float> hit_t, out_dev;
    // path tracing with the radiance cache
    ilg::DevBuf<uint32_t> train_slot, rec_of, s_meta, qry_meta;
    // hash-grid radiance cache (ILG_RENDER_HASH_CACHE)
    ilg::DevBuf<unsigned long long> hc_keys;
    ilg::DevBuf<float4> hc_vals;
    ilg::DevBuf<float> rec_feat, rec_tgt, qry_feat, qry_out;
    ilg::DevBuf<float4> rec_beta, qry_beta;
    uint32_t last_train_records = 0;
    bool last_hash_update = false;  // the last cached render updated the hash-grid cache
    float last_train_loss = 0.f;
    uint32_t last_render_launches = 0;
    // work counters of the last render made with ILG_RENDER_COUNT
    ilg::DevBuf<unsigned long long> render_stats;
    // path counter of the one-launch renderer (ILG_RENDER_PERSISTENT)
    ilg::DevBuf<unsigned long long> persist_next;
    bool counted = false;
    // the last frame's instantiated CUDA graph and the launch configuration it was captured for
    cudaGraphExec_t graph_exec = nullptr;
    std::vector<unsigned char> graph_key;
    uint32_t graph_kernels = 0;
    void drop_graph()
    {
        if (graph_exec) cudaGraphExecDestroy(graph_exec);
        graph_exec = nullptr;
        graph_key.clear();
    }

    // radiance-cache network
    ilg::DevBuf<float> mlp_w, mlp_m, mlp_v, mlp_grad, mlp_loss, mlp_raw, mlp_tgt, mlp_out;
    ilg::DevBuf<float> mlp_grid, mlp_grid_grad, mlp_grid_m, mlp_grid_v;
    ilg::DevBuf<uint32_t> mlp_enc;
    ilg::DevBuf<__nv_bfloat16> mlp_wf, mlp_wb, mlp_wu, mlp_wv, mlp_xcm, mlp_hcm, mlp_dzcm;
    bool mlp_ready = false;
    uint32_t mlp_encoding = 0;  // ILG_MLP_ENC_*
    uint32_t mlp_step = 0;
    float mlp_lr = 1e-2f;

    ilg::MlpDev mlp_view() const
    {
        ilg::MlpDev M;
        memset(&M, 0, sizeof(M));  // zero padding: the struct's bytes key the cached render graph
        M.w = mlp_w.ptr; M.m = mlp_m.ptr; M.v = mlp_v.ptr; M.grad = mlp_grad.ptr; M.loss = mlp_loss.ptr;
        M.wf = mlp_wf.ptr; M.wb = mlp_wb.ptr; M.wu = mlp_wu.ptr; M.wv = mlp_wv.ptr; M.err = derr.ptr; M.xcm = mlp_xcm.ptr; M.hcm = mlp_hcm.ptr; M.dzcm = mlp_dzcm.ptr;
        M.cap = (uint32_t)(mlp_xcm.cap / ilg::kMlpIn);
        M.grid = mlp_grid.ptr; M.grid_grad = mlp_grid_grad.ptr; M.grid_m = mlp_grid_m.ptr; M.grid_v = mlp_grid_v.ptr;
        ilg::grid_resolution(M.grid_res);
        M.encoding = mlp_encoding;
        // the frequency-only encoding has no grid columns to precompute
        M.enc = mlp_encoding == ilg::kEncHashGrid ? mlp_enc.ptr : nullptr;
        M.enc_cap = M.enc ? (uint32_t)(mlp_enc.cap / ilg::kGridLevels) : 0u;
        return M;
    }

    ilg::SceneView view() const
    {
        return ilg::SceneView{bb.nodes, bb.tris, bb.prim_of, stats.n_nodes, stats.n_tris};
    }

    int check_device_error()
    {
        uint32_t h = 0;
        if (cudaMemcpyAsync(&h, derr.ptr, sizeof(h), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
            cudaStreamSynchronize(stream) != cudaSuccess) {
            snprintf(err, sizeof(err), "reading the device error word failed");
            return ILG_ECUDA;
        }
        if (h) {
            cudaMemsetAsync(derr.ptr, 0, sizeof(uint32_t), stream);
            snprintf(err, sizeof(err), "device reported error flags 0x%x (bit0: traversal stack bound, bit1: node/triangle index out of range, bit2: node visit budget)", h);
            return ILG_EOVERFLOW;
        }
        return ILG_OK;
    }

    void release_all()
    {
        drop_graph();
        pos.release(); idx.release(); mat.release();
        bb.release_all();
        raw_tris.release(); raw_ready = false; render_stats.release(); persist_next.release();
        post_acc.release(); post_in.release(); post_out.release(); post_scratch.release();
        post_pixels = post_frames = 0;
        ro.release(); rd.release(); hprim.release(); ht.release(); hu.release(); hv.release(); hocc.release();
        derr.release(); dstats.release();
        mats.release(); lights.release(); light_range.release(); tri_attr.release(); light_of_prim.release();
        q_o0.release(); q_d0.release(); q_o1.release(); q_d1.release(); beta.release(); s_o.release();
        s_d.release(); s_c.release(); accum.release(); accum_direct.release(); accum_albedo.release(); q_p0.release(); q_p1.release(); counts.release();
        hit_tri.release(); hit_t.release(); out_dev.release(); path_scene.release(); s_sid.release();
        scene_table.release();
        train_slot.release(); rec_of.release(); s_meta.release(); qry_meta.release(); rec_feat.release();
        hc_keys.release(); hc_vals.release();
        rec_tgt.release();
        qry_feat.release(); qry_out.release(); rec_beta.release(); qry_beta.release();
        mlp_w.release(); mlp_m.release(); mlp_v.release(); mlp_grad.release(); mlp_loss.release();
        mlp_grid.release(); mlp_grid_grad.release(); mlp_grid_m.release(); mlp_grid_v.release(); mlp_enc.release();
        mlp_raw.release(); mlp_tgt.release(); mlp_out.release(); mlp_wf.release(); mlp_wb.release(); mlp_wu.release(); mlp_wv.release();
        mlp_xcm.release(); mlp_hcm.release(); mlp_dzcm.release();
    }
};
