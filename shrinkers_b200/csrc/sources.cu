// Sources in ascending order on the device, for the methods that need them
// (the treecode builds over the sorted spectrum, chebcode.rs:1088-1097; the
// NUFFT splat gathers contiguous source runs per grid cell).  Sortedness is
// checked on the device (or taken from the host check of a host-pointer
// call's upload); only unsorted input is sorted (CUB radix sort into library
// scratch).  The first and last entries IN THE CALLER'S ORDER are
// returned too: the NUFFT takes its grid bounds from them (nufft.rs:139-146).
#include "common.cuh"
#include "internal.h"

#include <cub/device/device_radix_sort.cuh>

namespace shrk {
namespace {

__global__ void unsorted_kernel(const double* __restrict__ src, int64_t n, int* flag) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (i < n && !(src[i - 1] <= src[i])) *flag = 1;
}

__global__ void iota_kernel(int* v, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] = (int)i;
}

// Device-side sortedness check (scratch slot 27 holds the flag) and the
// first / last entries, read back with one synchronisation.
shrk_status check_sorted(const double* d_src, int64_t ns, bool* sorted, double* first,
                         double* last, cudaStream_t s) {
  // A host-pointer call has checked its upload on the host already.
  if (source_hint(d_src, ns, sorted, first, last)) {
    if (!*sorted && ns > (int64_t)INT32_MAX) {
      set_error("unsorted input larger than 2^31 values: sort it before the call");
      return SHRK_EINVAL;
    }
    return SHRK_OK;
  }
  void* f = nullptr;
  SHRK_TRY(scratch_get(27, 256, &f));
  int* flag = (int*)f;
  SHRK_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), s));
  if (ns > 1) {
    LaunchScope ls("sources_check", s);
    unsorted_kernel<<<(unsigned)((ns - 1 + 255) / 256), 256, 0, s>>>(d_src, ns, flag);
    SHRK_CUDA(cudaGetLastError());
  }
  int h_flag = 0;
  SHRK_CUDA(cudaMemcpyAsync(&h_flag, flag, sizeof(int), cudaMemcpyDeviceToHost, s));
  SHRK_CUDA(cudaMemcpyAsync(first, d_src, sizeof(double), cudaMemcpyDeviceToHost, s));
  SHRK_CUDA(cudaMemcpyAsync(last, d_src + (ns - 1), sizeof(double), cudaMemcpyDeviceToHost, s));
  SHRK_CUDA(cudaStreamSynchronize(s));
  *sorted = h_flag == 0;
  if (!*sorted && ns > (int64_t)INT32_MAX) {
    set_error("unsorted input larger than 2^31 values: sort it before the call");
    return SHRK_EINVAL;
  }
  return SHRK_OK;
}

}  // namespace

// Scratch: slot 8 the sorted copy, slot 28 CUB's temporary.
shrk_status sorted_sources(const double* d_src, int64_t ns, const double** d_sorted,
                           double* first, double* last, cudaStream_t s) {
  bool sorted = true;
  SHRK_TRY(check_sorted(d_src, ns, &sorted, first, last, s));
  if (sorted) {
    *d_sorted = d_src;
    return SHRK_OK;
  }
  void* out = nullptr;
  SHRK_TRY(scratch_get(8, sizeof(double) * (size_t)ns, &out));
  size_t temp_bytes = 0;
  SHRK_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, temp_bytes, d_src, (double*)out, (int)ns, 0,
                                           64, s));
  void* temp = nullptr;
  SHRK_TRY(scratch_get(28, std::max<size_t>(temp_bytes, 256), &temp));
  {
    LaunchScope ls("sources_sort", s);
    SHRK_CUDA(cub::DeviceRadixSort::SortKeys(temp, temp_bytes, d_src, (double*)out, (int)ns, 0,
                                             64, s));
  }
  *d_sorted = (const double*)out;
  return SHRK_OK;
}

// As sorted_sources, with the source index of every sorted entry (scratch
// slot 29 holds the identity and the permutation).
shrk_status sorted_sources_perm(const double* d_src, int64_t ns, const double** d_sorted,
                                const int** d_perm, cudaStream_t s, double* lo, double* hi) {
  bool sorted = true;
  double first = 0.0, last = 0.0;
  SHRK_TRY(check_sorted(d_src, ns, &sorted, &first, &last, s));
  *d_perm = nullptr;
  if (sorted) {
    *d_sorted = d_src;
    if (lo) *lo = first;
    if (hi) *hi = last;
    return SHRK_OK;
  }
  void* pv = nullptr;
  SHRK_TRY(scratch_get(29, sizeof(int) * 2 * (size_t)ns, &pv));
  int* ids = (int*)pv;
  int* perm = ids + ns;
  iota_kernel<<<(unsigned)((ns + 255) / 256), 256, 0, s>>>(ids, ns);
  SHRK_CUDA(cudaGetLastError());
  add_launches(1);
  void* out = nullptr;
  SHRK_TRY(scratch_get(8, sizeof(double) * (size_t)ns, &out));
  size_t temp_bytes = 0;
  SHRK_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, d_src, (double*)out, ids, perm,
                                            (int)ns, 0, 64, s));
  void* temp = nullptr;
  SHRK_TRY(scratch_get(28, std::max<size_t>(temp_bytes, 256), &temp));
  {
    LaunchScope ls("sources_sort", s);
    SHRK_CUDA(cub::DeviceRadixSort::SortPairs(temp, temp_bytes, d_src, (double*)out, ids, perm,
                                              (int)ns, 0, 64, s));
  }
  *d_sorted = (const double*)out;
  *d_perm = perm;
  bool hs = false;
  double hf = 0.0, hl = 0.0;
  if ((lo || hi) && source_hint(d_src, ns, &hs, &hf, &hl, lo, hi)) return SHRK_OK;
  if (lo || hi) {
    double ends[2];
    SHRK_CUDA(cudaMemcpyAsync(&ends[0], out, sizeof(double), cudaMemcpyDeviceToHost, s));
    SHRK_CUDA(cudaMemcpyAsync(&ends[1], (const double*)out + (ns - 1), sizeof(double),
                              cudaMemcpyDeviceToHost, s));
    SHRK_CUDA(cudaStreamSynchronize(s));
    if (lo) *lo = ends[0];
    if (hi) *hi = ends[1];
  }
  return SHRK_OK;
}

}  // namespace shrk
