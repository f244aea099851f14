// prim.cuh -- device-wide primitives of libsexgpu (see prim.cu).
#pragma once
#include <cstddef>
#include <cuda_runtime.h>

namespace sx {
size_t scan_temp_ints(long long n);
void exclusive_scan(const int *in, int *out, long long n, int *total, int *tmp, cudaStream_t st,
                    const int *n_dev = nullptr);
int scan_launches(long long n);
size_t radix_temp_ints(long long n);
void radix_sort_pairs(unsigned *keys, unsigned *vals, unsigned *kalt, unsigned *valt, long long n,
                      int keybits, int *tmp, cudaStream_t st, const int *n_dev = nullptr,
                      unsigned *vfinal = nullptr, int *posmap = nullptr);
int radix_launches(int keybits, long long n);
}  // namespace sx
