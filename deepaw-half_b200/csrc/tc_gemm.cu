// Complex FP32 GEMM on the sm_100a tensor cores (tcgen05) for the mixed
// mode, on operands split into bf16 hi/lo planes.
//
// Every operand is first split, by a bandwidth-bound pass (presplit_kernel),
// or once per k point for the projector matrix, into four bf16 planes
// (Re hi, Re lo, Im hi, Im lo; x_hi = bf16(x), x_lo = bf16(x - x_hi)) stored
// in global memory in the tile layout of the tensor core, so that the tile of
// one stage is one contiguous bulk copy per plane.  One CTA then computes a
// 128 x BN tile of C (BN <= 256, a multiple of 16) over a range of k blocks
// (split-K when the tile grid alone cannot fill the GPU):
//   warp 8     one thread: per stage, waits for the stage to be free and
//              issues the eight bulk copies (cp.async.bulk, no multicast)
//              that fill it, completing on the stage's full mbarrier;
//   warp 9     one thread: per stage, the 12 tcgen05.mma of the three-term
//              split complex product into two TMEM accumulators
//                Re += Ar_h Br_h + Ar_h Br_l + Ar_l Br_h - (Ai_h Bi_h + Ai_h Bi_l + Ai_l Bi_h)
//                Im += Ar_h Bi_h + Ar_h Bi_l + Ar_l Bi_h + Ai_h Br_h + Ai_h Br_l + Ai_l Br_h
//              (the minus through the instruction descriptor's negate-A bit),
//              committing each stage back to the producer;
//   warps 0-7  the epilogue: tcgen05.ld of the accumulators, alpha / beta,
//              stores (or split-K partial sums).
// As many stages as fit the shared memory (up to eight) keep the copies
// ahead of the tensor core.  Every wait is bounded (tc.cuh): a stuck
// pipeline raises the runtime's error flag instead of hanging the GPU, and
// the CTA lets its copies and MMAs in flight land before it leaves.
//
// Plane layout (bytes), K-major canonical no-swizzle UMMA layout:
//   (r, k) of a 16-wide k block: (r/8) 256 + (k/8) 128 + (r%8) 16 + (k%8) 2,
//   LBO 128, SBO 256; in global memory k block kb of a plane starts at
//   kb rows_pad 32, so rows r0 .. r0 + R - 1 of it are R 32 contiguous bytes.
#include <cuda_bf16.h>

#include <algorithm>
#include <string>
#include <vector>

#include "tc.cuh"
#include "tc_gemm.h"
#include "tune.h"

namespace hb {

namespace {

using namespace tc;

constexpr int kBM = 128;
constexpr int kBK = 16;
constexpr int kMaxPipe = 8;          // stages: as many as fit the shared memory, up to this
constexpr size_t kSmemBudget = 225 * 1024;   // dynamic shared memory the stages may use
constexpr int kEpiWarps = 8;
constexpr int kProducerWarp = kEpiWarps, kMmaWarp = kEpiWarps + 1;
constexpr int kThreads = (kEpiWarps + 2) * 32;
constexpr int kSmemSlack = 1024;

__host__ __device__ inline uint32_t stage_bytes(int bn) {
  const uint32_t s = 4u * uint32_t(kBM) * 32u + 4u * uint32_t(bn) * 32u;
  return ((s + 1023u) / 1024u) * 1024u;
}

struct Out {
  int mode;          // 0: complex FP32 C, 1: complex FP64 C, 2: split-K partial sums
  void* c;
  void* c2;
  int split_col;
  long long ldc;
  double2 alpha, beta;
  int M, N;
};

// Two values at once (packed cvt.rn.bf16x2.f32): hi = (bf16(a), bf16(b)),
// lo = (bf16(a - hi.a), bf16(b - hi.b)), first value in the low half.
__device__ __forceinline__ void split_pair(float a, float b, uint32_t& hi, uint32_t& lo) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  const float2 hf = __bfloat1622float2(h);
  const __nv_bfloat162 l = __floats2bfloat162_rn(a - hf.x, b - hf.y);
  hi = *reinterpret_cast<const uint32_t*>(&h);
  lo = *reinterpret_cast<const uint32_t*>(&l);
}

__device__ __forceinline__ void unpack_g(int gp, double kf0, double kf1, double kf2, double& g0, double& g1,
                                         double& g2) {
  g0 = double((gp << 22) >> 22) + kf0;
  g1 = double((gp << 12) >> 22) + kf1;
  g2 = double((gp << 2) >> 22) + kf2;
}

// (cos, sin) of 2 pi (q.R / 2 pi) for one atom, reduced to one turn in FP64.
__device__ __forceinline__ void atom_phase(const double* __restrict__ afrac, int atom, double g0, double g1,
                                           double g2, float& c, float& s) {
  const double t = g0 * __ldg(afrac + 3 * atom) + g1 * __ldg(afrac + 3 * atom + 1) + g2 * __ldg(afrac + 3 * atom + 2);
  const float fr = float(t - rint(t));
  sincospif(2.0f * fr, &s, &c);
}

// Projector element for column `col` at plane wave g (g0..g2 = n + k), conj
// or not; `atom_c` caches the phase of the last atom seen.
__device__ __forceinline__ float2 projector_value(const TcOperand& op, int col, int g, double g0, double g1, double g2,
                                                  bool conj, int& atom_c, float& c, float& s) {
  const int d = __ldg(op.pcol + col);
  const int atom = d >> 16, frow = (d >> 2) & 0x3FFF, l = d & 3;
  if (atom != atom_c) {
    atom_phase(op.afrac, atom, g0, g1, g2, c, s);
    atom_c = atom;
  }
  const float f = __ldg(op.ftab + (long long)frow * op.npw + g);
  // conj(B) = f i^l (c + i s);  B = f (-i)^l (c - i s)
  float re, im;
  if (conj) {
    switch (l) {
      case 0: re = c; im = s; break;
      case 1: re = -s; im = c; break;
      case 2: re = -c; im = -s; break;
      default: re = s; im = -c; break;
    }
  } else {
    switch (l) {
      case 0: re = c; im = -s; break;
      case 1: re = -s; im = -c; break;
      case 2: re = -c; im = s; break;
      default: re = s; im = c; break;
    }
  }
  return make_float2(f * re, f * im);
}

// Pre-split planes of an operand.  Element (r, k) of op(.) (zero outside the
// matrix, r < rows_pad, k < 16 nkb) goes to the four bf16 planes, plane p at
// out + p plane_bytes, in the layout described at the top of this file.
// One thread per (row, 8 consecutive k): consecutive threads take consecutive
// rows, so row-contiguous operands load coalesced and each group of 8 rows
// stores 128 contiguous bytes per plane.  Projector operands generate their
// elements from the tables (kProj: row = plane wave, k = projector column;
// kProjConj: row = projector column, k = plane wave).
__global__ void presplit_kernel(TcOperand op, int rows_pad, int nkb, unsigned char* __restrict__ out,
                                long long plane_bytes) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)rows_pad * nkb * 2) return;
  const int r = int(t % rows_pad);
  const long long o = t / rows_pad;
  const int kb = int(o >> 1), half = int(o & 1), k0 = int(o * 8);
  float2 v[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = make_float2(0.f, 0.f);
  if (r < op.rows) {
    if (op.kind == TcOperand::kProj) {
      double g0, g1, g2;
      unpack_g(__ldg(op.gpack + r), op.kf0, op.kf1, op.kf2, g0, g1, g2);
      int atom_c = -1;
      float c = 0.f, s = 0.f;
#pragma unroll
      for (int i = 0; i < 8; ++i)
        if (k0 + i < op.kdim) v[i] = projector_value(op, k0 + i, r, g0, g1, g2, false, atom_c, c, s);
    } else if (op.kind == TcOperand::kProjConj) {
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int g = k0 + i;
        if (g < op.kdim) {
          double g0, g1, g2;
          unpack_g(__ldg(op.gpack + g), op.kf0, op.kf1, op.kf2, g0, g1, g2);
          int atom_c = -1;
          float c = 0.f, s = 0.f;
          v[i] = projector_value(op, r, g, g0, g1, g2, true, atom_c, c, s);
        }
      }
    } else {
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int k = k0 + i;
        if (k < op.kdim) {
          float2 x;
          if (op.kind == TcOperand::kDenseK) {
            const float2* src = r < op.split ? op.p + (long long)r * op.ld : op.p2 + (long long)(r - op.split) * op.ld;
            x = __ldg(src + k);
          } else {
            x = __ldg(op.p + r + (long long)k * op.ld);
          }
          if (op.conj) x.y = -x.y;
          v[i] = x;
        }
      }
    }
  }
  uint32_t w[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    split_pair(v[2 * i].x, v[2 * i + 1].x, w[0][i], w[1][i]);
    split_pair(v[2 * i].y, v[2 * i + 1].y, w[2][i], w[3][i]);
  }
  const long long off = (long long)kb * rows_pad * 32 + (long long)(r >> 3) * 256 + half * 128 + (r & 7) * 16;
#pragma unroll
  for (int p = 0; p < 4; ++p)
    *reinterpret_cast<uint4*>(out + p * plane_bytes + off) = make_uint4(w[p][0], w[p][1], w[p][2], w[p][3]);
}

// (A plane, B plane, accumulator 0 = Re / 1 = Im, negate A)
__constant__ int kCombo[12][4] = {{0, 0, 0, 0}, {0, 1, 0, 0}, {1, 0, 0, 0}, {2, 2, 0, 1}, {2, 3, 0, 1}, {3, 2, 0, 1},
                                  {0, 2, 1, 0}, {0, 3, 1, 0}, {1, 2, 1, 0}, {2, 0, 1, 0}, {2, 1, 1, 0}, {3, 0, 1, 0}};

template <typename T>
__device__ __forceinline__ void write_out(T* dst, double re, double im, const Out& o) {
  double ore = o.alpha.x * re - o.alpha.y * im, oim = o.alpha.x * im + o.alpha.y * re;
  if (o.beta.x != 0.0 || o.beta.y != 0.0) {
    const T old = *dst;
    ore += o.beta.x * double(old.x) - o.beta.y * double(old.y);
    oim += o.beta.x * double(old.y) + o.beta.y * double(old.x);
  }
  T v;
  v.x = decltype(v.x)(ore);
  v.y = decltype(v.y)(oim);
  *dst = v;
}

// A and B are pre-split planes (TcOperand::kPlanes); A.rows_pad >= gridDim.x
// 128 and B.rows_pad >= gridDim.y bn, both with nkb_total k blocks.
__global__ void __launch_bounds__(kThreads, 1)
    tc_cgemm_kernel(TcOperand A, TcOperand B, int bn, int nst, int kb_per_split, int nkb_total, Out out, int* err) {
  extern __shared__ __align__(1024) unsigned char smem_dyn[];
  __shared__ uint64_t full_bar[kMaxPipe], empty_bar[kMaxPipe], accum_bar;
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * bn, split = blockIdx.z;
  const int kb0 = split * kb_per_split;
  const int nkb = min(nkb_total, kb0 + kb_per_split) - kb0;
  const uint32_t sbase = (smem_addr(smem_dyn) + uint32_t(kSmemSlack - 1)) & ~uint32_t(kSmemSlack - 1);
  const uint32_t a_ps = uint32_t(kBM) * 32u, b_ps = uint32_t(bn) * 32u;
  const uint32_t sbytes = stage_bytes(bn);
  uint32_t tcols = 32;
  while (tcols < uint32_t(2 * bn)) tcols <<= 1;
  const uint32_t ci_off = tcols >> 1;
  volatile int* abort = &abort_flag;

  if (warp == kMmaWarp) tmem_alloc(&tmem_slot, tcols);
  if (threadIdx.x == 0) {
    for (int s = 0; s < nst; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    mbar_init(&accum_bar, 1);
    abort_flag = 0;
    mbar_init_fence();
  }
  tcgen05_fence_before();
  __syncthreads();
  tcgen05_fence_after();
  const uint32_t tmem = tmem_slot;

  if (warp == kProducerWarp) {
    if (lane == 0) {
      int issued = 0;
      for (int i = 0; i < nkb; ++i) {
        const int s = i % nst;
        if (i >= nst && !mbar_wait(&empty_bar[s], ((i / nst) - 1) & 1, abort)) break;
        const uint32_t abase = sbase + uint32_t(s) * sbytes, bbase = abase + 4u * a_ps;
        const long long kb = kb0 + i;
        mbar_expect_tx(&full_bar[s], 4u * (a_ps + b_ps));
#pragma unroll
        for (int p = 0; p < 4; ++p) {
          bulk_copy_g2s(abase + uint32_t(p) * a_ps, A.planes + p * A.plane_bytes + (kb * A.rows_pad + m0) * 32, a_ps,
                        &full_bar[s]);
          bulk_copy_g2s(bbase + uint32_t(p) * b_ps, B.planes + p * B.plane_bytes + (kb * B.rows_pad + n0) * 32, b_ps,
                        &full_bar[s]);
        }
        mbar_arrive(&full_bar[s]);
        issued = i + 1;
      }
      if (*abort) {   // let the copies still in flight land before the CTA leaves
        for (int i = max(0, issued - nst); i < issued; ++i) mbar_wait_drain(&full_bar[i % nst], (i / nst) & 1);
      }
    }
  } else if (warp == kMmaWarp) {
    if (lane == 0) {
      const uint32_t id_pos = instr_desc_bf16(bn, false, false, false), id_neg = instr_desc_bf16(bn, true, false, false);
      for (int i = 0; i < nkb; ++i) {
        const int s = i % nst;
        if (!mbar_wait(&full_bar[s], (i / nst) & 1, abort)) break;
        tcgen05_fence_after();
        const uint32_t abase = sbase + uint32_t(s) * sbytes, bbase = abase + 4u * a_ps;
#pragma unroll
        for (int c = 0; c < 12; ++c) {
          const uint64_t ad = smem_desc(abase + uint32_t(kCombo[c][0]) * a_ps, 128u, 256u);
          const uint64_t bd = smem_desc(bbase + uint32_t(kCombo[c][1]) * b_ps, 128u, 256u);
          mma_bf16(tmem + (kCombo[c][2] ? ci_off : 0u), ad, bd, kCombo[c][3] ? id_neg : id_pos,
                   i > 0 || (c != 0 && c != 6));
        }
        mma_commit(&empty_bar[s]);
      }
      mma_commit(&accum_bar);   // also on abort: arrives once every issued MMA has completed
    }
  } else {
    // epilogue: warp w reads TMEM lanes 32 (w % 4) .. +31, every other 16-column chunk
    const bool done = __all_sync(0xffffffffu, mbar_wait_drain(&accum_bar, 0));
    if (done && !*abort) {
      tcgen05_fence_after();
      const int q = warp & 3, half = warp >> 2;
      const int row = m0 + q * 32 + lane;
      for (int c = half; c < bn / 16; c += 2) {
        float cr[16], ci[16];
        const uint32_t ta = tmem + (uint32_t(q * 32) << 16) + uint32_t(c * 16);
        tmem_ld16(ta, cr);
        tmem_ld16(ta + ci_off, ci);
        tmem_ld_wait();
        if (row < out.M) {
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const int col = n0 + c * 16 + j;
            if (col >= out.N) break;
            if (out.mode == 2) {
              float2* w = reinterpret_cast<float2*>(out.c) + (long long)split * out.M * out.N + row +
                          (long long)col * out.M;
              *w = make_float2(cr[j], ci[j]);
            } else {
              const bool second = col >= out.split_col;
              const long long o = row + (long long)(second ? col - out.split_col : col) * out.ldc;
              if (out.mode == 0)
                write_out(reinterpret_cast<float2*>(second ? out.c2 : out.c) + o, cr[j], ci[j], out);
              else
                write_out(reinterpret_cast<double2*>(second ? out.c2 : out.c) + o, cr[j], ci[j], out);
            }
          }
        }
      }
    } else if (!done) {
      *abort = 1;
    }
  }
  tcgen05_fence_before();
  __syncthreads();
  if (warp == kMmaWarp) {
    tcgen05_fence_after();
    tmem_dealloc(tmem, tcols);
  }
  if (threadIdx.x == 0 && abort_flag) atomicExch(err, 1);
}

template <typename T>
__global__ void splitk_reduce_kernel(const float2* __restrict__ W, int S, int M, int N, double2 alpha, double2 beta,
                                     T* C, T* C2, int split_col, long long ldc) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)M * N) return;
  const int i = int(t % M), j = int(t / M);
  double sr = 0.0, si = 0.0;
  for (int s = 0; s < S; ++s) {
    const float2 w = W[(long long)s * M * N + t];
    sr += w.x;
    si += w.y;
  }
  const bool second = j >= split_col;
  T* dst = (second ? C2 : C) + i + (long long)(second ? j - split_col : j) * ldc;
  Out o{};
  o.alpha = alpha;
  o.beta = beta;
  write_out(dst, sr, si, o);
}

int pick_bn(int N) {
  const int nt = (N + 255) / 256;
  int bn = (N + nt - 1) / nt;
  bn = ((bn + 15) / 16) * 16;
  return std::min(256, std::max(16, bn));
}

}  // namespace

TcOperand tc_dense_a(cublasOperation_t op, const float2* A, long long lda, int M, int K) {
  TcOperand o;
  o.kind = op == CUBLAS_OP_N ? TcOperand::kDenseMN : TcOperand::kDenseK;
  o.conj = op == CUBLAS_OP_C;
  o.rows = M;
  o.kdim = K;
  o.p = A;
  o.ld = lda;
  return o;
}

TcOperand tc_dense_b(cublasOperation_t op, const float2* B, long long ldb, int K, int N) {
  TcOperand o;
  o.kind = op == CUBLAS_OP_N ? TcOperand::kDenseK : TcOperand::kDenseMN;
  o.conj = op == CUBLAS_OP_C;
  o.rows = N;
  o.kdim = K;
  o.p = B;
  o.ld = ldb;
  return o;
}

void tc_cgemm(Runtime& rt, const TcOperand& A, const TcOperand& B, int M, int N, int K, double2 alpha,
              double2 beta, void* C, bool c_fp64, long long ldc, void* C2, int split_col) {
  if (M <= 0 || N <= 0) return;
  cudaStream_t st = rt.stream;
  if (rt.tc_err.size() == 0) {
    rt.tc_err.resize(1);
    rt.tc_err.zero(st);
  }
  if (C2 == nullptr) split_col = INT_MAX;
  // The split-K boundaries follow from the default tile width only, so the
  // tile width the autotuner picks (tune.h) changes no result.
  const int bn0 = pick_bn(N);
  const int mt = (M + kBM - 1) / kBM, nt0 = (N + bn0 - 1) / bn0;
  const int nkb = (K + kBK - 1) / kBK;
  int dev = 0, sms = 148;
  HALF_CUDA(cudaGetDevice(&dev));
  HALF_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const long long tiles = (long long)mt * nt0;
  int splits = 1;
  if (tiles < sms && nkb > 0) {
    splits = int(std::min<long long>((sms + tiles - 1) / tiles, std::max(1, nkb / 4)));
    splits = std::max(1, splits);
  }
  const int kbps = nkb > 0 ? (nkb + splits - 1) / splits : 0;
  if (nkb > 0) splits = (nkb + kbps - 1) / kbps;
  // tile width: 0, 1 or 2 more N tiles than the fewest are the candidates
  std::vector<int> cand;
  for (int extra = 0; extra < 3; ++extra) {
    const int t = nt0 + extra, w = ((N + t - 1) / t + 15) / 16 * 16;
    if (w >= 16 && (cand.empty() || w < cand.back())) cand.push_back(w);
  }
  int tune_token = 0, bn = bn0;
  if (nkb > 0 && cand.size() > 1) {
    const std::string key = "gemm " + std::to_string(A.kind) + std::to_string(B.kind) + " " + std::to_string(M) +
                            "x" + std::to_string(N) + "x" + std::to_string(K) + " s" + std::to_string(splits);
    const int idx = Tuner::pick(key, cand);
    bn = cand[idx];
    tune_token = Tuner::begin(key, idx, st);
  }
  const int nt = (N + bn - 1) / bn;
  // Operands not given as planes are split into bf16 planes in global memory
  // by a bandwidth-bound pass; the GEMM feeds its stages by bulk copies.
  TcOperand Ak = A, Bk = B;
  Profile& pf = rt.prof;
  int span0 = -1;
  if (nkb > 0) {
    const int rpa = mt * kBM, rpb = nt * bn;
    auto check = [&](const TcOperand& o, int rp, const char* which) {
      if (o.kind == TcOperand::kPlanes &&
          (o.planes == nullptr || o.rows_pad < rp || o.rows_pad % 16 != 0 || o.kdim != K ||
           o.plane_bytes < (long long)o.rows_pad * nkb * 32 || (reinterpret_cast<uintptr_t>(o.planes) & 15) != 0))
        fail(kInvalidArgument, std::string("pre-split ") + which + " operand does not cover the product");
    };
    check(A, rpa, "A");
    check(B, rpb, "B");
    const long long pa = A.kind != TcOperand::kPlanes ? (long long)rpa * nkb * 32 : 0;
    const long long pb = B.kind != TcOperand::kPlanes ? (long long)rpb * nkb * 32 : 0;
    if (pa + pb > 0) {
      const size_t bytes = size_t(4) * size_t(pa + pb);
      if (rt.tc_planes.size() < bytes) rt.tc_planes.resize(bytes);
      unsigned char* planes = rt.tc_planes.get();
      span0 = pf.record(st);
      if (pa > 0) {
        const long long th = (long long)rpa * nkb * 2;
        presplit_kernel<<<ceil_div(th, 256), 256, 0, st>>>(A, rpa, nkb, planes, pa);
        Ak = TcOperand();
        Ak.kind = TcOperand::kPlanes;
        Ak.rows = A.rows;
        Ak.kdim = A.kdim;
        Ak.planes = planes;
        Ak.plane_bytes = pa;
        Ak.rows_pad = rpa;
        ++pf.launches;
      }
      if (pb > 0) {
        const long long th = (long long)rpb * nkb * 2;
        presplit_kernel<<<ceil_div(th, 256), 256, 0, st>>>(B, rpb, nkb, planes + 4 * pa, pb);
        Bk = TcOperand();
        Bk.kind = TcOperand::kPlanes;
        Bk.rows = B.rows;
        Bk.kdim = B.kdim;
        Bk.planes = planes + 4 * pa;
        Bk.plane_bytes = pb;
        Bk.rows_pad = rpb;
        ++pf.launches;
      }
      HALF_LAUNCH("tensor-core operand split");
    }
  }
  const size_t sbytes = stage_bytes(bn);
  const int nst = int(std::min<size_t>(kMaxPipe, (kSmemBudget - kSmemSlack) / sbytes));
  if (nst < 2) fail(kInternal, "tensor-core GEMM stage does not fit shared memory twice");
  const size_t smem = size_t(nst) * sbytes + kSmemSlack;
  raise_smem_limit(tc_cgemm_kernel, smem);
  Out o{};
  o.alpha = alpha;
  o.beta = beta;
  o.M = M;
  o.N = N;
  const bool direct = splits == 1 && nkb > 0;
  if (direct) {
    o.mode = c_fp64 ? 1 : 0;
    o.c = C;
    o.c2 = C2;
    o.split_col = split_col;
    o.ldc = ldc;
  } else {
    const size_t bytes = size_t(std::max(splits, 1)) * M * N * sizeof(float2);
    if (rt.tc_work.size() < bytes) rt.tc_work.resize(bytes);
    o.mode = 2;
    o.c = rt.tc_work.get();
  }
  if (nkb > 0) {
    const int e0 = span0 >= 0 ? span0 : pf.record(st);
    tc_cgemm_kernel<<<dim3(mt, nt, splits), kThreads, smem, st>>>(Ak, Bk, bn, nst, kbps, nkb, o, rt.tc_err.get());
    HALF_LAUNCH("tensor-core cgemm");
    Tuner::finish(tune_token, st, 1.0);
    pf.span(Profile::kTensor, e0, pf.record(st));
    pf.tensor_flops += 24.0 * double(M) * double(N) * double(K);
    ++pf.tensor_launches;
    ++pf.launches;
  }
  if (!direct) {
    const long long mn = (long long)M * N;
    const int S = nkb > 0 ? splits : 0;
    const float2* W = reinterpret_cast<const float2*>(rt.tc_work.get());
    if (c_fp64)
      splitk_reduce_kernel<double2><<<ceil_div(mn, 256), 256, 0, st>>>(W, S, M, N, alpha, beta,
                                                                       static_cast<double2*>(C),
                                                                       static_cast<double2*>(C2), split_col, ldc);
    else
      splitk_reduce_kernel<float2><<<ceil_div(mn, 256), 256, 0, st>>>(W, S, M, N, alpha, beta,
                                                                      static_cast<float2*>(C),
                                                                      static_cast<float2*>(C2), split_col, ldc);
    HALF_LAUNCH("split-K reduction");
    ++rt.prof.launches;
  }
}

TcOperand tc_presplit_a(Runtime& rt, const TcOperand& op, DeviceBuffer<unsigned char>& store) {
  if (op.kind == TcOperand::kPlanes) fail(kInvalidArgument, "operand is already split");
  const int rows_pad = (op.rows + kBM - 1) / kBM * kBM, nkb = (op.kdim + kBK - 1) / kBK;
  const long long pbytes = (long long)rows_pad * nkb * 32;
  TcOperand o;
  o.kind = TcOperand::kPlanes;
  o.rows = op.rows;
  o.kdim = op.kdim;
  o.rows_pad = rows_pad;
  o.plane_bytes = pbytes;
  if (pbytes == 0) return o;
  if (store.size() < size_t(4 * pbytes)) store.resize(size_t(4 * pbytes));
  presplit_kernel<<<ceil_div((long long)rows_pad * nkb * 2, 256), 256, 0, rt.stream>>>(op, rows_pad, nkb, store.get(),
                                                                                       pbytes);
  HALF_LAUNCH("tensor-core operand split (kept)");
  ++rt.prof.launches;
  o.planes = store.get();
  return o;
}

void tc_check(Runtime& rt) {
  if (rt.tc_err.size() == 0) return;
  int flag = 0;
  HALF_CUDA(cudaMemcpyAsync(&flag, rt.tc_err.get(), sizeof(int), cudaMemcpyDeviceToHost, rt.stream));
  HALF_CUDA(cudaStreamSynchronize(rt.stream));
  if (flag) {
    rt.tc_err.zero(rt.stream);
    fail(kInternal, "tensor-core GEMM pipeline wait timed out");
  }
}

}  // namespace hb
