// Device side of half_solve_kpoint_mapped: the eigenvectors are reordered
// from HALF's G order into the host code's order (src/half_c_api.F90:521-588
// does this on the host, element by element) by one gather kernel, so the
// eigenvector block crosses PCIe once, already in the caller's layout.
#include "context.h"

namespace hb {

namespace {

// dst[b*ld + j] = src[b*n + src_row[j]] for j < n, zero for n <= j < ld
__global__ void gather_rows_kernel(const double2* __restrict__ src, long long n, int nb,
                                   const int* __restrict__ src_row, double2* __restrict__ dst, long long ld) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= ld * nb) return;
  const int b = int(t / ld);
  const long long j = t - (long long)b * ld;
  dst[t] = j < n ? src[(long long)b * n + src_row[j]] : make_double2(0.0, 0.0);
}

}  // namespace

void gather_rows_to_host(Runtime& rt, const double2* src, long long n, int nb, const std::vector<int>& src_row,
                         long long ld, double2* host_dst) {
  DeviceBuffer<int> rows;
  rows.upload(src_row, rt.stream);
  DeviceBuffer<double2> dst(size_t(ld) * nb);
  gather_rows_kernel<<<ceil_div(ld * nb, 256), 256, 0, rt.stream>>>(src, n, nb, rows.get(), dst.get(), ld);
  HALF_LAUNCH("mapped gather");
  rt.prof.launches += 1;
  HALF_CUDA(cudaMemcpyAsync(host_dst, dst.get(), size_t(ld) * nb * sizeof(double2), cudaMemcpyDeviceToHost,
                            rt.stream));
  HALF_CUDA(cudaStreamSynchronize(rt.stream));
}

}  // namespace hb
