// compat_lib.cu -- libsexgpu_compat.so: the whole libsexgpu plus the
// reference's thirteen CUDA entry points (include/sexgpu_compat.h).
#include "sexgpu.cu"
#include "compat.cu"
