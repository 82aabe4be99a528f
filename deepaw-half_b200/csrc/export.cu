// VASP wave-coefficient export on the device (src/half_vaspwave.F90:94-154):
// the eigenvectors of each k point in VASP's plane-wave order (the box's
// x-fastest order, vasp_permutation :143-154) as interleaved single-precision
// (re, im), band-major -- the layout of /wave/spin_1/kpoint_<k>/wave
// [nb][npw][2] that the reference's HDF5 bridge writes.  One gather-convert
// kernel per k point; the permutation is a host sort of the basis's box
// indices.
#include <algorithm>
#include <numeric>

#include "context.h"

namespace hb {

namespace {

// out[b*npw + g] = (float re, float im) of vec[b*ld + order[g]]; the float
// conversion rounds to nearest like the reference's real(., c_float).
__global__ void pack_vasp_kernel(const double2* __restrict__ vec, long long ld, int npw, int nb,
                                 const int* __restrict__ order, float2* __restrict__ out) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)npw * nb) return;
  const int b = int(t / npw), g = int(t - (long long)b * npw);
  const double2 c = vec[(long long)b * ld + order[g]];
  out[t] = make_float2(__double2float_rn(c.x), __double2float_rn(c.y));
}

}  // namespace

std::vector<int> vasp_order(const Basis& b) {
  const long long nx = b.shape[0], ny = b.shape[1], nz = b.shape[2];
  std::vector<long long> key(b.npw());
  for (long long i = 0; i < b.npw(); ++i) {
    const long long c = b.fft_index[i], gx = c / (ny * nz), r = c - gx * ny * nz, gy = r / nz, gz = r - gy * nz;
    key[i] = gx + nx * (gy + ny * gz);
  }
  std::vector<int> order(b.npw());
  std::iota(order.begin(), order.end(), 0);
  std::sort(order.begin(), order.end(), [&](int x, int y) { return key[x] < key[y]; });
  return order;
}

void pack_vasp_device(Runtime& rt, const double2* vec, long long ld, int npw, int nb, const std::vector<int>& order,
                      float2* out) {
  cudaStream_t s = rt.stream;
  DeviceBuffer<int> dorder;
  dorder.upload(order, s);
  const long long total = (long long)npw * nb;
  if (total > 0) {
    pack_vasp_kernel<<<ceil_div(total, 256), 256, 0, s>>>(vec, ld, npw, nb, dorder.get(), out);
    HALF_LAUNCH("pack vasp waves");
  }
  HALF_CUDA(cudaStreamSynchronize(s));   // dorder is released on return
}

}  // namespace hb
