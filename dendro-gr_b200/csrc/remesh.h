// Remesh indicator: exact wavelet test, block features, BF16 MLP.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace bssn {

struct MeshState;

// parameters of the 16 -> 64 -> 64 -> 1 MLP: W1, b1, W2, b2, W3, b3
constexpr int MLP_NPARAM = 64 * 16 + 64 + 64 * 64 + 64 + 64 + 1;

// one element (octant) of a block
struct ElemRef {
    int32_t blk;
    int16_t o[3];
    int16_t pad;
};

int remesh_elements(MeshState* m);
int launch_wavelet_scores(MeshState* m, const double* const* U, int nvars, double* scores,
                          const uint8_t* need, cudaStream_t s);
int launch_block_flags(MeshState* m, const double* scores, int nvars, double tol, double* ratio,
                       uint8_t* flags, const uint8_t* need, cudaStream_t s);
int launch_features(MeshState* m, const double* const* U, float* feats, cudaStream_t s);
// per-element features (n_elems x 16)
int launch_element_features(MeshState* m, const double* const* U, float* feats, cudaStream_t s);
// exact test on the elements with need_e set (off: n_elems + 1, list: n_elems
// scratch entries, count: one)
int launch_wavelet_elements(MeshState* m, const double* const* U, int nvars, double* scores,
                            const uint8_t* need_e, int64_t* off, int64_t* count, int32_t* list,
                            cudaStream_t s);
// per-element decision with block settling (remesh_settle_elem_kernel)
int launch_remesh_select_elem(MeshState* m, const float* lr, const float* lk, float lo_r, float hi_r,
                              float lo_k, float hi_k, double audit_frac, uint64_t seed, uint8_t* need_e,
                              uint8_t* decided_e, int* stats, cudaStream_t s);
int launch_remesh_merge_elem(MeshState* m, const uint8_t* need_e, const uint8_t* decided_e,
                             const double* scores, int nvars, double tol, double keep_fac, const float* lr,
                             const float* lk, float lo_r, float lo_k, int* stats, uint8_t* flags_r,
                             uint8_t* flags_k, cudaStream_t s);
// tensor-core forward (BF16 operands, FP32 accumulation); the decisions use it
int launch_mlp_fwd(const void* wq, const float* norm, const float* X, int n, float* logits,
                   cudaStream_t s);
// the same network with FP32 activations on the FP32 pipes (the training
// kernel's forward)
int launch_mlp_fwd_fp32(const void* wq, const float* norm, const float* X, int n, float* logits,
                        cudaStream_t s);
size_t mlp_grad_scratch_floats(int n);
int launch_mlp_grad(const void* wq, const float* norm, const float* X, const float* Y,
                    const float* C, int n, float* grad, float* loss, float* scratch,
                    cudaStream_t s);
int launch_adam(float* master, void* wq, const float* grad, float* m, float* v, float lr,
                float b1, float b2, float eps, int t, cudaStream_t s);
int launch_remesh_select(const float* logits, int nblk, float lo, float hi, double audit_frac,
                         uint64_t seed, uint8_t* need, uint8_t* decided, int* stats,
                         cudaStream_t s);
int launch_remesh_merge(int nblk, const uint8_t* need, const uint8_t* decided,
                        const uint8_t* exact, const float* logits, float lo, int* stats,
                        uint8_t* flags, cudaStream_t s);

int launch_remesh_select2(const float* lr, const float* lk, int nblk, float lo_r, float hi_r,
                          float lo_k, float hi_k, double audit_frac, uint64_t seed, uint8_t* need,
                          uint8_t* decided, int* stats, cudaStream_t s);
int launch_remesh_merge2(int nblk, const uint8_t* need, const uint8_t* decided, const double* ratio,
                         double keep_fac, const float* lr, const float* lk, float lo_r, float lo_k,
                         int* stats, uint8_t* flags_r, uint8_t* flags_k, cudaStream_t s);

}  // namespace bssn
