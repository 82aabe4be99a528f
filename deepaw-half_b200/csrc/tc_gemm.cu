// Complex FP32 GEMM on the sm_100a tensor cores (tcgen05), with the mixed
// mode's operands split into bf16 hi/lo planes inside the kernel.
//
// One CTA computes a 128 x BN tile of C (BN <= 256, a multiple of 16) over a
// range of k blocks (split-K when the tile grid alone cannot fill the GPU).
//   warps 0-7  producers: read a 128 x 16 slice of op(A) and a BN x 16 slice
//              of op(B) per stage (dense complex FP32 from global memory, or
//              projector elements generated from their tables), split every
//              real and imaginary part into x_hi = bf16(x), x_lo =
//              bf16(x - x_hi) and store the four planes (Re hi, Re lo,
//              Im hi, Im lo) of each operand in the canonical no-swizzle
//              UMMA layout; then, after the last stage, the epilogue
//              (tcgen05.ld of the accumulators, alpha / beta, stores);
//   warp 8     one thread issues, per stage, the 12 tcgen05.mma of the
//              three-term split complex product into two TMEM accumulators
//                Re += Ar_h Br_h + Ar_h Br_l + Ar_l Br_h - (Ai_h Bi_h + Ai_h Bi_l + Ai_l Bi_h)
//                Im += Ar_h Bi_h + Ar_h Bi_l + Ar_l Bi_h + Ai_h Br_h + Ai_h Br_l + Ai_l Br_h
//              (the minus through the instruction descriptor's negate-A bit)
//              and commits each stage back to the producers.
// Up to eight stages of mbarrier-synchronised shared-memory buffers (as many
// as fit) overlap the loads with the tensor core.  Every wait is bounded (tc.cuh): a stuck
// pipeline raises the runtime's error flag instead of hanging the GPU.
//
// Shared-memory plane layouts (bytes; the producers choose the layout that
// lets a warp's stores hit 32 distinct banks):
//   K-major  (r, k): (r/8) 256 + (k/8) 128 + (r%8) 16 + (k%8) 2   LBO 128, SBO 256
//   MN-major (r, k): (r/8) 272 + (k/8) 128 + (k%8) 16 + (r%8) 2   LBO 128, SBO 272
// Consecutive planes are staggered by 64 bytes so that one store instruction
// writing a hi plane (even lanes) and a lo plane (odd lanes) is conflict-free.
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
constexpr int kProdWarps = 8;
constexpr int kProdThreads = kProdWarps * 32;
constexpr int kThreads = kProdThreads + 32;
constexpr int kSmemSlack = 128;

__host__ __device__ inline bool is_mn(int kind) {
  return kind == TcOperand::kDenseMN || kind == TcOperand::kProjConj;
}
__host__ __device__ inline uint32_t plane_stride(int rows, bool mn) {
  const uint32_t bytes = uint32_t(rows / 8) * (mn ? 272u : 256u);
  return ((bytes + 127u) / 128u) * 128u + 64u;
}
__host__ __device__ inline uint32_t stage_bytes(int bn, int akind, int bkind) {
  const uint32_t s = 4u * plane_stride(kBM, is_mn(akind)) + 4u * plane_stride(bn, is_mn(bkind));
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

// Splits this lane's element and stores, with its neighbour (lane ^ 1), one
// 4-byte pair per plane: even lanes the hi planes, odd lanes the lo planes.
// The pair's first element is the even lane's.  Every lane must call this.
__device__ __forceinline__ void store_pair(float2 v, int lane, uint32_t base, uint32_t pstride, uint32_t off,
                                           bool store) {
  uint32_t hi, lo;   // (Re, Im) hi parts and lo parts
  split_pair(v.x, v.y, hi, lo);
  const bool even = (lane & 1) == 0;
  const uint32_t recv = __shfl_xor_sync(0xffffffffu, even ? lo : hi, 1);
  const uint32_t own = even ? hi : lo;
  const uint32_t a = even ? own : recv, b = even ? recv : own;
  if (store) {
    const uint32_t pr = even ? 0u : 1u;
    st_shared_u32(base + pr * pstride + off, __byte_perm(a, b, 0x5410));
    st_shared_u32(base + (pr + 2u) * pstride + off, __byte_perm(a, b, 0x7632));
  }
}

// Dense operands are filled in two halves so the producer loop can issue
// the global loads of stage i + 1 before it splits and stores stage i:
// load_dense_* brings this warp's elements of one slice into registers (zero
// outside the matrix), store_dense_* splits and stores them.  NV is the
// register count per lane: 8 for the 128-row A slice, 16 for B (up to 256 rows).

// k contiguous: each warp step covers 4 rows x 8 k.
template <int NV>
__device__ __forceinline__ void load_dense_k(const TcOperand& op, int r0, int R, int k0, int warp, int lane,
                                             float2 (&v)[NV]) {
  const int nsteps = (R >> 2) * 2;
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    const int t = warp + i * kProdWarps;
    v[i] = make_float2(0.f, 0.f);
    if (t < nsteps) {
      const int r = r0 + (t >> 1) * 4 + (lane >> 3), k = k0 + (t & 1) * 8 + (lane & 7);
      if (r < op.rows && k < op.kdim) {
        const float2* src = r < op.split ? op.p + (long long)r * op.ld : op.p2 + (long long)(r - op.split) * op.ld;
        v[i] = __ldg(src + k);
      }
    }
  }
}

template <int NV>
__device__ __forceinline__ void store_dense_k(const TcOperand& op, int R, uint32_t base, uint32_t pstride, int warp,
                                              int lane, const float2 (&v)[NV]) {
  const int nsteps = (R >> 2) * 2;
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    const int t = warp + i * kProdWarps;
    if (t < nsteps) {
      const int r = (t >> 1) * 4 + (lane >> 3), kl = (t & 1) * 8 + (lane & 7);
      float2 x = v[i];
      if (op.conj) x.y = -x.y;
      const uint32_t off = uint32_t(r >> 3) * 256u + uint32_t(t & 1) * 128u + uint32_t(r & 7) * 16u +
                           uint32_t((kl & 7) >> 1) * 4u;
      store_pair(x, lane, base, pstride, off, true);
    }
  }
}

// rows contiguous: each warp step covers 32 rows at one k.
template <int NV>
__device__ __forceinline__ void load_dense_mn(const TcOperand& op, int r0, int R, int k0, int warp, int lane,
                                              float2 (&v)[NV]) {
  const int nsteps = ((R + 31) >> 5) * 16;
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    const int t = warp + i * kProdWarps;
    v[i] = make_float2(0.f, 0.f);
    if (t < nsteps) {
      const int rl = (t >> 4) * 32 + lane, r = r0 + rl, k = k0 + (t & 15);
      if (rl < R && r < op.rows && k < op.kdim) v[i] = __ldg(op.p + r + (long long)k * op.ld);
    }
  }
}

template <int NV>
__device__ __forceinline__ void store_dense_mn(const TcOperand& op, int R, uint32_t base, uint32_t pstride, int warp,
                                               int lane, const float2 (&v)[NV]) {
  const int nsteps = ((R + 31) >> 5) * 16;
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    const int t = warp + i * kProdWarps;
    if (t < nsteps) {
      const int rl = (t >> 4) * 32 + lane, kl = t & 15, rp = rl & ~1;
      float2 x = v[i];
      if (op.conj) x.y = -x.y;
      const uint32_t off = uint32_t(rp >> 3) * 272u + uint32_t(kl >> 3) * 128u + uint32_t(kl & 7) * 16u +
                           uint32_t((rp & 7) >> 1) * 4u;
      store_pair(x, lane, base, pstride, off, rl < R);
    }
  }
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

// Eight generated elements -> four 16-byte plane chunks at `off`.
__device__ __forceinline__ void store_chunk8(const float2 (&v)[8], uint32_t base, uint32_t pstride, uint32_t off) {
  uint32_t w[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    split_pair(v[2 * i].x, v[2 * i + 1].x, w[0][i], w[1][i]);
    split_pair(v[2 * i].y, v[2 * i + 1].y, w[2][i], w[3][i]);
  }
#pragma unroll
  for (int p = 0; p < 4; ++p) st_shared_v4(base + uint32_t(p) * pstride + off, w[p][0], w[p][1], w[p][2], w[p][3]);
}

// Pre-split planes of a dense operand.  Element (r, k) of op(.) (zero outside
// the matrix, r < rows_pad, k < 16 nkb) goes to the four bf16 planes (Re hi,
// Re lo, Im hi, Im lo), plane p at out + p plane_bytes, k block kb at
// kb rows_pad 32 bytes, and inside it the K-major core-matrix layout
// (r/8) 256 + (k/8) 128 + (r%8) 16 + (k%8) 2: the tile layout in shared
// memory, so the tile of any 8-aligned row range is ONE contiguous bulk copy.
// One thread per (row, 8 consecutive k): consecutive threads take consecutive
// rows, so row-contiguous operands load coalesced and each group of 8 rows
// stores 128 contiguous bytes per plane.
__global__ void presplit_kernel(TcOperand op, int rows_pad, int nkb, unsigned char* __restrict__ out,
                                long long plane_bytes) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)rows_pad * nkb * 2) return;
  const int r = int(t % rows_pad);
  const long long o = t / rows_pad;
  const int kb = int(o >> 1), half = int(o & 1), k0 = int(o * 8);
  float2 v[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int k = k0 + i;
    float2 x = make_float2(0.f, 0.f);
    if (r < op.rows && k < op.kdim) {
      if (op.kind == TcOperand::kDenseK) {
        const float2* src = r < op.split ? op.p + (long long)r * op.ld : op.p2 + (long long)(r - op.split) * op.ld;
        x = __ldg(src + k);
      } else {
        x = __ldg(op.p + r + (long long)k * op.ld);
      }
      if (op.conj) x.y = -x.y;
    }
    v[i] = x;
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

// conj(B)^T slice: rows = projector columns (MN-major chunks of 8), k = plane waves.
__device__ __forceinline__ void fill_proj_conj(const TcOperand& op, int r0, int R, int k0, uint32_t base,
                                               uint32_t pstride, int tid) {
  const int tasks = (R >> 3) * 16;
  for (int t = tid; t < tasks; t += kProdThreads) {
    const int pc = t >> 4, kl = t & 15, g = k0 + kl;
    float2 v[8];
    if (g < op.npw) {
      double g0, g1, g2;
      unpack_g(__ldg(op.gpack + g), op.kf0, op.kf1, op.kf2, g0, g1, g2);
      int atom_c = -1;
      float c = 0.f, s = 0.f;
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int col = r0 + pc * 8 + i;
        v[i] = col < op.rows ? projector_value(op, col, g, g0, g1, g2, true, atom_c, c, s) : make_float2(0.f, 0.f);
      }
    } else {
#pragma unroll
      for (int i = 0; i < 8; ++i) v[i] = make_float2(0.f, 0.f);
    }
    store_chunk8(v, base, pstride, uint32_t(pc) * 272u + uint32_t(kl >> 3) * 128u + uint32_t(kl & 7) * 16u);
  }
}

// B slice: rows = plane waves, k = projector columns (K-major chunks of 8).
__device__ __forceinline__ void fill_proj(const TcOperand& op, int r0, int R, int k0, uint32_t base,
                                          uint32_t pstride, int tid) {
  const int tasks = R * 2;
  for (int t = tid; t < tasks; t += kProdThreads) {
    const int row = t % R, kc = t / R, g = r0 + row;
    float2 v[8];
    if (g < op.rows) {
      double g0, g1, g2;
      unpack_g(__ldg(op.gpack + g), op.kf0, op.kf1, op.kf2, g0, g1, g2);
      int atom_c = -1;
      float c = 0.f, s = 0.f;
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int col = k0 + kc * 8 + i;
        v[i] = col < op.kdim ? projector_value(op, col, g, g0, g1, g2, false, atom_c, c, s) : make_float2(0.f, 0.f);
      }
    } else {
#pragma unroll
      for (int i = 0; i < 8; ++i) v[i] = make_float2(0.f, 0.f);
    }
    store_chunk8(v, base, pstride, uint32_t(row >> 3) * 256u + uint32_t(kc) * 128u + uint32_t(row & 7) * 16u);
  }
}

template <int NV>
__device__ __forceinline__ void load_operand(const TcOperand& op, int r0, int R, int k0, int warp, int lane,
                                             float2 (&v)[NV]) {
  if (op.kind == TcOperand::kDenseK) load_dense_k(op, r0, R, k0, warp, lane, v);
  else if (op.kind == TcOperand::kDenseMN) load_dense_mn(op, r0, R, k0, warp, lane, v);
}

// Generated operands compute their elements here; dense ones store the
// registers their load_operand brought in.
template <int NV>
__device__ __forceinline__ void store_operand(const TcOperand& op, int r0, int R, int k0, uint32_t base,
                                              uint32_t pstride, int warp, int lane, const float2 (&v)[NV]) {
  switch (op.kind) {
    case TcOperand::kDenseK: store_dense_k(op, R, base, pstride, warp, lane, v); break;
    case TcOperand::kDenseMN: store_dense_mn(op, R, base, pstride, warp, lane, v); break;
    case TcOperand::kProjConj: fill_proj_conj(op, r0, R, k0, base, pstride, warp * 32 + lane); break;
    case TcOperand::kProj: fill_proj(op, r0, R, k0, base, pstride, warp * 32 + lane); break;
    default: break;   // kPlanes: bulk copies fill the stage
  }
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
  const bool a_mn = is_mn(A.kind), b_mn = is_mn(B.kind);
  const uint32_t a_ps = plane_stride(kBM, a_mn), b_ps = plane_stride(bn, b_mn);
  const uint32_t sbytes = stage_bytes(bn, A.kind, B.kind);
  const uint32_t bulk_bytes = (A.kind == TcOperand::kPlanes ? 4u * kBM * 32u : 0u) +
                              (B.kind == TcOperand::kPlanes ? 4u * uint32_t(bn) * 32u : 0u);
  uint32_t tcols = 32;
  while (tcols < uint32_t(2 * bn)) tcols <<= 1;
  const uint32_t ci_off = tcols >> 1;
  volatile int* abort = &abort_flag;

  if (warp == kProdWarps) tmem_alloc(&tmem_slot, tcols);
  if (threadIdx.x == 0) {
    for (int s = 0; s < nst; ++s) {
      mbar_init(&full_bar[s], kProdWarps);
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

  if (warp < kProdWarps) {
    // software pipeline: the dense loads of stage i + 1 are in flight while
    // stage i is split and stored
    float2 va[2][8], vb[2][16];
    if (nkb > 0) {
      load_operand(A, m0, kBM, kb0 * kBK, warp, lane, va[0]);
      load_operand(B, n0, bn, kb0 * kBK, warp, lane, vb[0]);
    }
    for (int i = 0; i < nkb; i += 2) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int ii = i + h;
        if (ii < nkb) {
          if (ii + 1 < nkb) {
            load_operand(A, m0, kBM, (kb0 + ii + 1) * kBK, warp, lane, va[h ^ 1]);
            load_operand(B, n0, bn, (kb0 + ii + 1) * kBK, warp, lane, vb[h ^ 1]);
          }
          const int s = ii % nst;
          if (ii >= nst && !__all_sync(0xffffffffu, mbar_wait(&empty_bar[s], ((ii / nst) - 1) & 1, abort))) {
            i = nkb;   // leave both loops
            break;
          }
          const uint32_t abase = sbase + uint32_t(s) * sbytes, bbase = abase + 4u * a_ps;
          const int k0 = (kb0 + ii) * kBK;
          if (bulk_bytes && warp == 0 && lane == 0) {   // pre-split operands: one bulk copy per plane
            mbar_expect_tx(&full_bar[s], bulk_bytes);
            const long long kb = kb0 + ii;
            if (A.kind == TcOperand::kPlanes)
              for (int p = 0; p < 4; ++p)
                bulk_copy_g2s(abase + uint32_t(p) * a_ps,
                              A.planes + p * A.plane_bytes + kb * A.rows_pad * 32 + (long long)m0 * 32,
                              uint32_t(kBM * 32), &full_bar[s]);
            if (B.kind == TcOperand::kPlanes)
              for (int p = 0; p < 4; ++p)
                bulk_copy_g2s(bbase + uint32_t(p) * b_ps,
                              B.planes + p * B.plane_bytes + kb * B.rows_pad * 32 + (long long)n0 * 32,
                              uint32_t(bn * 32), &full_bar[s]);
          }
          store_operand(A, m0, kBM, k0, abase, a_ps, warp, lane, va[h]);
          store_operand(B, n0, bn, k0, bbase, b_ps, warp, lane, vb[h]);
          fence_proxy_async_smem();
          __syncwarp();
          if (lane == 0) mbar_arrive(&full_bar[s]);
        }
      }
    }
    // epilogue: warp w reads TMEM lanes 32 (w % 4) .. +31, every other 16-column chunk
    if (__all_sync(0xffffffffu, mbar_wait(&accum_bar, 0, abort))) {
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
    }
  } else if (lane == 0) {
    const uint32_t id_pos = instr_desc_bf16(bn, false, a_mn, b_mn), id_neg = instr_desc_bf16(bn, true, a_mn, b_mn);
    const uint32_t a_sbo = a_mn ? 272u : 256u, b_sbo = b_mn ? 272u : 256u;
    for (int i = 0; i < nkb; ++i) {
      const int s = i % nst;
      if (!mbar_wait(&full_bar[s], (i / nst) & 1, abort)) break;
      tcgen05_fence_after();
      const uint32_t abase = sbase + uint32_t(s) * sbytes, bbase = abase + 4u * a_ps;
#pragma unroll
      for (int c = 0; c < 12; ++c) {
        const uint64_t ad = smem_desc(abase + uint32_t(kCombo[c][0]) * a_ps, 128u, a_sbo);
        const uint64_t bd = smem_desc(bbase + uint32_t(kCombo[c][1]) * b_ps, 128u, b_sbo);
        mma_bf16(tmem + (kCombo[c][2] ? ci_off : 0u), ad, bd, kCombo[c][3] ? id_neg : id_pos,
                 i > 0 || (c != 0 && c != 6));
      }
      mma_commit(&empty_bar[s]);
    }
    mma_commit(&accum_bar);   // also on abort: arrives once every issued MMA has completed
  }
  tcgen05_fence_before();
  __syncthreads();
  if (warp == kProdWarps) {
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
  // Dense operands are split once into bf16 planes in global memory by a
  // bandwidth-bound pass; the GEMM then feeds its stages by bulk copies.
  // Generated projector operands keep their in-kernel producers.
  TcOperand Ak = A, Bk = B;
  Profile& pf = rt.prof;
  int span0 = -1;
  if (nkb > 0) {
    auto dense = [](const TcOperand& o) { return o.kind == TcOperand::kDenseK || o.kind == TcOperand::kDenseMN; };
    const int rpa = mt * kBM, rpb = nt * bn;
    const long long pa = dense(A) ? (long long)rpa * nkb * 32 : 0, pb = dense(B) ? (long long)rpb * nkb * 32 : 0;
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
  const size_t sbytes = stage_bytes(bn, Ak.kind, Bk.kind);
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
