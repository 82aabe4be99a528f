// Complex FP32 GEMM on the BF16 tensor cores (the mixed mode's large GEMMs).
//
// cuBLAS runs complex FP32 GEMMs (CGEMM) on SIMT kernels on B200 even with its
// BF16x9 emulation enabled.  Here op(A) = Ar + i Ai and op(B) = Br + i Bi are
// split into bf16 planes, x = x_hi + x_lo with x_hi = bf16(x) and
// x_lo = bf16(x - x_hi), and every real product is taken as
// x_hi y_hi + x_hi y_lo + x_lo y_hi (relative error about 2^-16, FP32
// accumulation).  With
//   A' = [Ar_hi Ar_hi Ar_lo Ai_hi Ai_hi Ai_lo]                  (M x 6K)
//   B' = [ Br_hi  Br_lo  Br_hi -Bi_hi -Bi_lo -Bi_hi ;           (6K x 2N)
//          Bi_hi  Bi_lo  Bi_hi  Br_hi  Br_lo  Br_hi ]^T-blocks
// one real BF16 GEMM A' B' gives [Re(op(A) op(B)) | Im(op(A) op(B))], and an
// epilogue forms C = alpha (Re + i Im) + beta C.
#include <cuda_bf16.h>

#include "blas.h"

namespace hb {

namespace {

__device__ __forceinline__ void split(float x, __nv_bfloat16& hi, __nv_bfloat16& lo) {
  hi = __float2bfloat16_rn(x);
  lo = __float2bfloat16_rn(x - __bfloat162float(hi));
}

// op(A) = A (M x K, lda): A' column-major M x 6K.
__global__ void pack_a_n_kernel(const float2* __restrict__ A, long long lda, int M, int K,
                                __nv_bfloat16* __restrict__ Ap) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)M * K) return;
  const int m = int(t % M), k = int(t / M);
  const float2 v = A[m + (long long)k * lda];
  __nv_bfloat16 rh, rl, ih, il;
  split(v.x, rh, rl);
  split(v.y, ih, il);
  const long long mk = (long long)M * K, o = m + (long long)k * M;
  Ap[o] = rh; Ap[o + mk] = rh; Ap[o + 2 * mk] = rl;
  Ap[o + 3 * mk] = ih; Ap[o + 4 * mk] = ih; Ap[o + 5 * mk] = il;
}

// op(A) = A^H or A^T (A is K x M, lda): A'^T column-major 6K x M.
__global__ void pack_a_t_kernel(const float2* __restrict__ A, long long lda, int M, int K, bool conj,
                                __nv_bfloat16* __restrict__ Ap) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)M * K) return;
  const int k = int(t % K), m = int(t / K);
  const float2 v = A[k + (long long)m * lda];
  __nv_bfloat16 rh, rl, ih, il;
  split(v.x, rh, rl);
  split(conj ? -v.y : v.y, ih, il);
  __nv_bfloat16* col = Ap + (long long)m * 6 * K + k;
  col[0] = rh; col[K] = rh; col[2 * (long long)K] = rl;
  col[3 * (long long)K] = ih; col[4 * (long long)K] = ih; col[5 * (long long)K] = il;
}

// op(B) = B (K x N, ldb): B' column-major 6K x 2N.
__global__ void pack_b_n_kernel(const float2* __restrict__ B, long long ldb, int K, int N,
                                __nv_bfloat16* __restrict__ Bp) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)K * N) return;
  const int k = int(t % K), n = int(t / K);
  const float2 v = B[k + (long long)n * ldb];
  __nv_bfloat16 rh, rl, ih, il;
  split(v.x, rh, rl);
  split(v.y, ih, il);
  const __nv_bfloat16 nih = __hneg(ih), nil = __hneg(il);
  __nv_bfloat16* re = Bp + (long long)n * 6 * K + k;
  __nv_bfloat16* im = Bp + ((long long)N + n) * 6 * K + k;
  re[0] = rh; re[K] = rl; re[2 * (long long)K] = rh;
  re[3 * (long long)K] = nih; re[4 * (long long)K] = nil; re[5 * (long long)K] = nih;
  im[0] = ih; im[K] = il; im[2 * (long long)K] = ih;
  im[3 * (long long)K] = rh; im[4 * (long long)K] = rl; im[5 * (long long)K] = rh;
}

// op(B) = B^H or B^T (B is N x K, ldb): B'^T column-major 2N x 6K.
__global__ void pack_b_t_kernel(const float2* __restrict__ B, long long ldb, int K, int N, bool conj,
                                __nv_bfloat16* __restrict__ Bp) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)K * N) return;
  const int n = int(t % N), k = int(t / N);
  const float2 v = B[n + (long long)k * ldb];
  __nv_bfloat16 rh, rl, ih, il;
  split(v.x, rh, rl);
  split(conj ? -v.y : v.y, ih, il);
  const __nv_bfloat16 nih = __hneg(ih), nil = __hneg(il);
  const long long ld = 2LL * N;
  __nv_bfloat16* re = Bp + n + (long long)k * ld;
  __nv_bfloat16* im = Bp + N + n + (long long)k * ld;
  const long long step = (long long)K * ld;
  re[0] = rh; re[step] = rl; re[2 * step] = rh; re[3 * step] = nih; re[4 * step] = nil; re[5 * step] = nih;
  im[0] = ih; im[step] = il; im[2 * step] = ih; im[3 * step] = rh; im[4 * step] = rl; im[5 * step] = rh;
}

// C = alpha (Cf[:, :N] + i Cf[:, N:]) + beta C
__global__ void split_epilogue_kernel(const float* __restrict__ Cf, int M, int N, float2 alpha, float2 beta,
                                      float2* __restrict__ C, long long ldc) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)M * N) return;
  const int m = int(t % M), n = int(t / M);
  const float re = Cf[m + (long long)n * M], im = Cf[m + ((long long)N + n) * M];
  float2 out = make_float2(alpha.x * re - alpha.y * im, alpha.x * im + alpha.y * re);
  float2* c = C + m + (long long)n * ldc;
  if (beta.x != 0.0f || beta.y != 0.0f) {
    const float2 old = *c;
    out.x += beta.x * old.x - beta.y * old.y;
    out.y += beta.x * old.y + beta.y * old.x;
  }
  *c = out;
}

template <typename T>
T* grow(DeviceBuffer<unsigned char>& b, size_t count) {
  const size_t bytes = count * sizeof(T);
  if (b.size() < bytes) b.resize(bytes);
  return reinterpret_cast<T*>(b.get());
}

}  // namespace

void gemm_c32_split(Runtime& rt, cublasOperation_t ta, cublasOperation_t tb, int M, int N, int K, float2 alpha,
                    const float2* A, long long lda, const float2* B, long long ldb, float2 beta, float2* C,
                    long long ldc) {
  cudaStream_t s = rt.stream;
  __nv_bfloat16* Ap = grow<__nv_bfloat16>(rt.split_a, size_t(6) * M * K);
  __nv_bfloat16* Bp = grow<__nv_bfloat16>(rt.split_b, size_t(12) * K * N);
  float* Cf = grow<float>(rt.split_c, size_t(2) * M * N);
  const long long mk = (long long)M * K, kn = (long long)K * N;
  if (ta == CUBLAS_OP_N) pack_a_n_kernel<<<ceil_div(mk, 256), 256, 0, s>>>(A, lda, M, K, Ap);
  else pack_a_t_kernel<<<ceil_div(mk, 256), 256, 0, s>>>(A, lda, M, K, ta == CUBLAS_OP_C, Ap);
  if (tb == CUBLAS_OP_N) pack_b_n_kernel<<<ceil_div(kn, 256), 256, 0, s>>>(B, ldb, K, N, Bp);
  else pack_b_t_kernel<<<ceil_div(kn, 256), 256, 0, s>>>(B, ldb, K, N, tb == CUBLAS_OP_C, Bp);
  HALF_LAUNCH("split packing");
  const float one = 1.0f, zero = 0.0f;
  cublas_check(cublasGemmEx(rt.blas, ta == CUBLAS_OP_N ? CUBLAS_OP_N : CUBLAS_OP_T,
                            tb == CUBLAS_OP_N ? CUBLAS_OP_N : CUBLAS_OP_T, M, 2 * N, 6 * K, &one, Ap, CUDA_R_16BF,
                            ta == CUBLAS_OP_N ? M : 6 * K, Bp, CUDA_R_16BF, tb == CUBLAS_OP_N ? 6 * K : 2 * N,
                            &zero, Cf, CUDA_R_32F, M, CUBLAS_COMPUTE_32F, CUBLAS_GEMM_DEFAULT),
               "bf16 split gemm");
  split_epilogue_kernel<<<ceil_div((long long)M * N, 256), 256, 0, s>>>(Cf, M, N, alpha, beta, C, ldc);
  HALF_LAUNCH("split epilogue");
  rt.prof.launches += 3;
}

}  // namespace hb
