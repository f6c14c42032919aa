// kernels.h -- launchers of the sm_100a kernels, called by the C++ engine.
//
// State layout in HBM: 2^n complex64 amplitudes (float2, re/im interleaved),
// 256-byte aligned, amplitude i <-> basis state with qubit q = bit q of i.
// All launchers are asynchronous on the given stream and return the launch
// status (cudaGetLastError after the launch).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace qlb {

struct Mat2f { float2 m[4]; };          // row-major 2x2 complex64

// ---- state set-up (state.cu) -------------------------------------------
cudaError_t launch_init_zero(float2* a, uint64_t dim, cudaStream_t s);
// complex128 (device staging) -> complex64 state slice
cudaError_t launch_c128_to_c64(const double2* src, float2* dst, uint64_t count, cudaStream_t s);
cudaError_t launch_c64_to_c128(const float2* src, double2* dst, uint64_t count, cudaStream_t s);
// out[i] = a[idx[i]] widened to complex128 (idx checked by the caller).
cudaError_t launch_gather(const float2* a, const uint64_t* idx, uint64_t count, double2* out, cudaStream_t s);

// ---- plain per-instruction kernels (gates.cu) ---------------------------
// Generic 2x2 on target t (one HBM sweep).
cudaError_t launch_apply_1q(float2* a, uint32_t n, uint32_t t, const Mat2f& m, cudaStream_t s);
// diag(d0, d1) on target t; when d0 == 1 only the |1> half is touched.
cudaError_t launch_apply_diag1(float2* a, uint32_t n, uint32_t t, float2 d0, float2 d1, cudaStream_t s);
// Swap a[base|ma] <-> a[base|mb] over all bases with zeros at the sorted
// hole positions h[0..nh-1] (CX, SWAP, CCX, CSWAP, GLOBAL_SWAP).
cudaError_t launch_swap_subspace(float2* a, uint32_t n, const uint32_t* holes, uint32_t nh,
                                 uint64_t ma, uint64_t mb, cudaStream_t s);
// Multiply a[i] by `ph` for every i with all bits of `mask` set (CZ, CP).
cudaError_t launch_phase_mask(float2* a, uint32_t n, const uint32_t* holes, uint32_t nh,
                              uint64_t mask, float2 ph, cudaStream_t s);
// Dense k-qubit unitary (k <= 6), FP32 on CUDA cores; `mat` is a device
// row-major 2^k x 2^k complex64 matrix, matrix bit j <-> qubit q[j].
cudaError_t launch_apply_dense(float2* a, uint32_t n, const uint32_t* q, uint32_t k,
                               const float2* mat, cudaStream_t s);

// ---- FP64 reductions / measurement / sampling (reduce.cu) ---------------
// Writes sum |a|^2 over all amplitudes (mask == 0) or over the amplitudes
// with bit `qubit` set, into *out (device double).
cudaError_t launch_norm_sq(const float2* a, uint64_t dim, double* partial, uint32_t partial_cap,
                           double* out, cudaStream_t s);
cudaError_t launch_prob_one(const float2* a, uint32_t n, uint32_t qubit, double* partial,
                            uint32_t partial_cap, double* out, cudaStream_t s);
// out[0] = sum |a|^2, out[1+q] = sum over amplitudes with bit q set.
cudaError_t launch_qubit_marginals(const float2* a, uint32_t n, double* partial, uint32_t partial_cap,
                                   double* out, cudaStream_t s);
uint32_t marginals_partial_size(uint32_t n);
// Zero the half with bit t != outcome, scale the other by `scale`.
cudaError_t launch_collapse(float2* a, uint32_t n, uint32_t t, int outcome, float scale, cudaStream_t s);
// Counter-based sampling of `shots` basis states; `chunk_sums` needs
// 2^(n - kSampleChunkLog2) doubles (when n > kSampleChunkLog2).
constexpr uint32_t kSampleChunkLog2 = 12;
cudaError_t launch_sample(const float2* a, uint32_t n, uint64_t seed, uint64_t shots, double* chunk_sums,
                          uint64_t* out, cudaStream_t s);
uint64_t sample_scratch_doubles(uint32_t n);

}  // namespace qlb
