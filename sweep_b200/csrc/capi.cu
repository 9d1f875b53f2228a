// capi.cu -- the extern "C" entry points declared in include/sweep_b200.h.
// Each one validates, dispatches on the equation family, and turns any error
// into (non-zero return, message) -- nothing is thrown across the boundary.
#include "acoustic2d.cuh"
#include "elastic2d.cuh"
#include "elastic3d.cuh"
#include "acoustic_orders.cuh"
#include "elastic_orders.cuh"
#include "vti2d.cuh"
#include "vti3d.cuh"

namespace sweep {
namespace a3d {
void sizes(const sweep_acoustic_desc*, int, int, int64_t*, int64_t*);
void forward(const sweep_acoustic_desc*, int, int, float*, void*, void*, int64_t, cudaStream_t);
void backward(const sweep_acoustic_desc*, int, int, const float*, const void*, float*, float*,
              float*, float*, void*, int64_t, cudaStream_t);
}  // namespace a3d
}  // namespace sweep

using namespace sweep;

extern "C" int sweep_b200_abi_version(void) { return SWEEP_B200_ABI_VERSION; }

extern "C" int sweep_b200_acoustic_sizes(const sweep_acoustic_desc* d, int32_t mem_mode, int32_t ckpt_every,
                                         int64_t* workspace_bytes, int64_t* tape_bytes,
                                         char* err, int32_t err_cap)
{
    return guarded(err, err_cap, [&] {
        SWEEP_REQUIRE(d && workspace_bytes && tape_bytes, "null argument");
        SWEEP_REQUIRE(d->ndim == 2 || d->ndim == 3, "acoustic: ndim %d is not built", d->ndim);
        if (d->M != 4) aord::sizes(d, mem_mode, ckpt_every, workspace_bytes, tape_bytes);
        else if (d->ndim == 2) a2d::sizes(d, mem_mode, ckpt_every, workspace_bytes, tape_bytes);
        else a3d::sizes(d, mem_mode, ckpt_every, workspace_bytes, tape_bytes);
    });
}

extern "C" int sweep_b200_acoustic_forward(const sweep_acoustic_desc* d, int32_t mem_mode, int32_t ckpt_every,
                                           float* record, void* tape, void* workspace, int64_t workspace_bytes,
                                           void* stream, char* err, int32_t err_cap)
{
    return guarded(err, err_cap, [&] {
        SWEEP_REQUIRE(d != nullptr, "null descriptor");
        SWEEP_REQUIRE(d->ndim == 2 || d->ndim == 3, "acoustic: ndim %d is not built", d->ndim);
        if (d->M != 4)
            aord::forward(d, mem_mode, ckpt_every, record, tape, workspace, workspace_bytes,
                          static_cast<cudaStream_t>(stream));
        else if (d->ndim == 2)
            a2d::forward(d, mem_mode, ckpt_every, record, tape, workspace, workspace_bytes,
                         static_cast<cudaStream_t>(stream));
        else
            a3d::forward(d, mem_mode, ckpt_every, record, tape, workspace, workspace_bytes,
                         static_cast<cudaStream_t>(stream));
    });
}

extern "C" int sweep_b200_acoustic_backward(const sweep_acoustic_desc* d, int32_t mem_mode, int32_t ckpt_every,
                                            const float* adj, const void* tape, float* grad_vp,
                                            float* grad_wavelet, float* illum_src, float* illum_rec,
                                            void* workspace, int64_t workspace_bytes, void* stream,
                                            char* err, int32_t err_cap)
{
    return guarded(err, err_cap, [&] {
        SWEEP_REQUIRE(d != nullptr, "null descriptor");
        SWEEP_REQUIRE(d->ndim == 2 || d->ndim == 3, "acoustic: ndim %d is not built", d->ndim);
        if (d->M != 4)
            aord::backward(d, mem_mode, ckpt_every, adj, tape, grad_vp, grad_wavelet, illum_src, illum_rec,
                           workspace, workspace_bytes, static_cast<cudaStream_t>(stream));
        else if (d->ndim == 2)
            a2d::backward(d, mem_mode, ckpt_every, adj, tape, grad_vp, grad_wavelet, illum_src, illum_rec,
                          workspace, workspace_bytes, static_cast<cudaStream_t>(stream));
        else
            a3d::backward(d, mem_mode, ckpt_every, adj, tape, grad_vp, grad_wavelet, illum_src, illum_rec,
                          workspace, workspace_bytes, static_cast<cudaStream_t>(stream));
    });
}

extern "C" int sweep_b200_elastic_sizes(const sweep_elastic_desc* d, int32_t mem_mode, int32_t ckpt_every,
                                        int64_t* workspace_bytes, int64_t* tape_bytes, char* err, int32_t err_cap)
{
    return guarded(err, err_cap, [&] {
        SWEEP_REQUIRE(d && workspace_bytes && tape_bytes, "null argument");
        if (d->M != 4) eord::sizes(d, mem_mode, ckpt_every, workspace_bytes, tape_bytes);
        else el2d::sizes(d, mem_mode, ckpt_every, workspace_bytes, tape_bytes);
    });
}

extern "C" int sweep_b200_elastic_forward(const sweep_elastic_desc* d, int32_t mem_mode, int32_t ckpt_every,
                                          float* record, void* tape, void* workspace, int64_t workspace_bytes,
                                          void* stream, char* err, int32_t err_cap)
{
    return guarded(err, err_cap, [&] {
        SWEEP_REQUIRE(d != nullptr, "null descriptor");
        if (d->M != 4)
            eord::forward(d, mem_mode, ckpt_every, record, tape, workspace, workspace_bytes,
                          static_cast<cudaStream_t>(stream));
        else
            el2d::forward(d, mem_mode, ckpt_every, record, tape, workspace, workspace_bytes,
                          static_cast<cudaStream_t>(stream));
    });
}

extern "C" int sweep_b200_elastic_backward(const sweep_elastic_desc* d, int32_t mem_mode, int32_t ckpt_every,
                                           const float* adj, const void* tape, float* grad_vp, float* grad_vs,
                                           float* grad_rho, void* workspace, int64_t workspace_bytes,
                                           void* stream, char* err, int32_t err_cap)
{
    return guarded(err, err_cap, [&] {
        SWEEP_REQUIRE(d != nullptr, "null descriptor");
        if (d->M != 4)
            eord::backward(d, mem_mode, ckpt_every, adj, tape, grad_vp, grad_vs, grad_rho, workspace,
                           workspace_bytes, static_cast<cudaStream_t>(stream));
        else
            el2d::backward(d, mem_mode, ckpt_every, adj, tape, grad_vp, grad_vs, grad_rho, workspace,
                           workspace_bytes, static_cast<cudaStream_t>(stream));
    });
}

extern "C" int sweep_b200_vti_sizes(const sweep_vti_desc* d, int32_t mem_mode, int32_t ckpt_every,
                                    int64_t* workspace_bytes, int64_t* tape_bytes, char* err, int32_t err_cap)
{
    return guarded(err, err_cap, [&] {
        SWEEP_REQUIRE(d && workspace_bytes && tape_bytes, "null argument");
        vti::sizes(d, mem_mode, ckpt_every, workspace_bytes, tape_bytes);
    });
}

extern "C" int sweep_b200_vti_forward(const sweep_vti_desc* d, int32_t mem_mode, int32_t ckpt_every, float* record,
                                      void* tape, void* workspace, int64_t workspace_bytes, void* stream, char* err,
                                      int32_t err_cap)
{
    return guarded(err, err_cap, [&] {
        SWEEP_REQUIRE(d != nullptr, "null descriptor");
        vti::forward(d, mem_mode, ckpt_every, record, tape, workspace, workspace_bytes,
                     static_cast<cudaStream_t>(stream));
    });
}

extern "C" int sweep_b200_vti_backward(const sweep_vti_desc* d, int32_t mem_mode, int32_t ckpt_every,
                                       const float* adj, const void* tape, float* grad_vp, float* grad_epsilon,
                                       float* grad_delta, float* grad_rho, void* workspace, int64_t workspace_bytes,
                                       void* stream, char* err, int32_t err_cap)
{
    return guarded(err, err_cap, [&] {
        SWEEP_REQUIRE(d != nullptr, "null descriptor");
        vti::backward(d, mem_mode, ckpt_every, adj, tape, grad_vp, grad_epsilon, grad_delta, grad_rho, workspace,
                      workspace_bytes, static_cast<cudaStream_t>(stream));
    });
}

extern "C" int sweep_b200_vti3d_sizes(const sweep_vti3d_desc* d, int32_t mem_mode, int32_t ckpt_every,
                                      int64_t* workspace_bytes, int64_t* tape_bytes, char* err, int32_t err_cap)
{
    return guarded(err, err_cap, [&] {
        SWEEP_REQUIRE(d && workspace_bytes && tape_bytes, "null argument");
        vti3::sizes(d, mem_mode, ckpt_every, workspace_bytes, tape_bytes);
    });
}

extern "C" int sweep_b200_vti3d_forward(const sweep_vti3d_desc* d, int32_t mem_mode, int32_t ckpt_every,
                                        float* record, void* tape, void* workspace, int64_t workspace_bytes,
                                        void* stream, char* err, int32_t err_cap)
{
    return guarded(err, err_cap, [&] {
        SWEEP_REQUIRE(d != nullptr, "null descriptor");
        vti3::forward(d, mem_mode, ckpt_every, record, tape, workspace, workspace_bytes,
                      static_cast<cudaStream_t>(stream));
    });
}

extern "C" int sweep_b200_vti3d_backward(const sweep_vti3d_desc* d, int32_t mem_mode, int32_t ckpt_every,
                                         const float* adj, const void* tape, float* grad_vp, float* grad_epsilon,
                                         float* grad_delta, float* grad_rho, void* workspace,
                                         int64_t workspace_bytes, void* stream, char* err, int32_t err_cap)
{
    return guarded(err, err_cap, [&] {
        SWEEP_REQUIRE(d != nullptr, "null descriptor");
        vti3::backward(d, mem_mode, ckpt_every, adj, tape, grad_vp, grad_epsilon, grad_delta, grad_rho, workspace,
                       workspace_bytes, static_cast<cudaStream_t>(stream));
    });
}

extern "C" int sweep_b200_elastic3d_sizes(const sweep_elastic3d_desc* d, int32_t mem_mode, int32_t ckpt_every,
                                          int64_t* workspace_bytes, int64_t* tape_bytes, char* err, int32_t err_cap)
{
    return guarded(err, err_cap, [&] {
        SWEEP_REQUIRE(d && workspace_bytes && tape_bytes, "null argument");
        el3d::sizes(d, mem_mode, ckpt_every, workspace_bytes, tape_bytes);
    });
}

extern "C" int sweep_b200_elastic3d_forward(const sweep_elastic3d_desc* d, int32_t mem_mode, int32_t ckpt_every,
                                            float* record, void* tape, void* workspace, int64_t workspace_bytes,
                                            void* stream, char* err, int32_t err_cap)
{
    return guarded(err, err_cap, [&] {
        SWEEP_REQUIRE(d != nullptr, "null descriptor");
        el3d::forward(d, mem_mode, ckpt_every, record, tape, workspace, workspace_bytes,
                      static_cast<cudaStream_t>(stream));
    });
}

extern "C" int sweep_b200_elastic3d_backward(const sweep_elastic3d_desc* d, int32_t mem_mode, int32_t ckpt_every,
                                             const float* adj, const void* tape, float* grad_vp, float* grad_vs,
                                             float* grad_rho, void* workspace, int64_t workspace_bytes,
                                             void* stream, char* err, int32_t err_cap)
{
    return guarded(err, err_cap, [&] {
        SWEEP_REQUIRE(d != nullptr, "null descriptor");
        el3d::backward(d, mem_mode, ckpt_every, adj, tape, grad_vp, grad_vs, grad_rho, workspace,
                       workspace_bytes, static_cast<cudaStream_t>(stream));
    });
}
