// k_fits.cu -- FITS pixel data to the float32 frame on the device.
//
// The file's data block is copied to the device as it is stored (big-endian,
// BITPIX bytes per pixel) and converted here, as read_body
// (src/fits/fitsbody.c:195) converts it on the host: integer pixels
// (BITPIX 8 unsigned, 16 and 32 signed) become value * BSCALE + BZERO in
// float with BSCALE and BZERO first rounded to float, and a pixel equal to
// BLANK becomes -BIG; BITPIX -32 pixels with an all-ones exponent (Inf, NaN)
// become -BIG, the others value * BSCALE + BZERO in float; BITPIX -64 the
// same test on the double's exponent, the product and sum in double and one
// rounding to float.
#include "common.cuh"
#include "kernels.cuh"

namespace sx {

constexpr float FITS_BLANK = -1e+30f;  // -BIG as a pixel value

__device__ __forceinline__ unsigned fits_bswap32(unsigned x) { return __byte_perm(x, 0, 0x0123); }

template <int BITPIX>
__global__ void k_fits_to_float(const unsigned char *__restrict__ raw, float *__restrict__ out, long long n, float bs,
                                float bz, int has_blank, long long blank) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        float v;
        if (BITPIX == 8) {
            const unsigned char c = raw[i];
            v = (has_blank && c == (unsigned char)blank) ? FITS_BLANK : c * bs + bz;
        } else if (BITPIX == 16) {
            const unsigned short u = reinterpret_cast<const unsigned short *>(raw)[i];
            const short s = (short)(unsigned short)((u >> 8) | (u << 8));
            v = (has_blank && s == (short)blank) ? FITS_BLANK : s * bs + bz;
        } else if (BITPIX == 32) {
            const int s = (int)fits_bswap32(reinterpret_cast<const unsigned *>(raw)[i]);
            v = (has_blank && s == (int)blank) ? FITS_BLANK : s * bs + bz;
        } else if (BITPIX == -32) {
            const unsigned u = fits_bswap32(reinterpret_cast<const unsigned *>(raw)[i]);
            v = ((u & 0x7f800000u) == 0x7f800000u) ? FITS_BLANK : __uint_as_float(u) * bs + bz;
        } else {
            const uint2 q = reinterpret_cast<const uint2 *>(raw)[i];
            const unsigned hi = fits_bswap32(q.x), lo = fits_bswap32(q.y);
            const double d = __hiloint2double((int)hi, (int)lo);
            v = ((hi & 0x7ff00000u) == 0x7ff00000u) ? FITS_BLANK : (float)(d * (double)bs + (double)bz);
        }
        out[i] = v;
    }
}

// false for an unknown BITPIX
bool launch_fits_to_float(const void *d_raw, int bitpix, double bscale, double bzero, int has_blank,
                          long long blank, float *d_out, long long n, cudaStream_t st) {
    const float bs = (float)bscale, bz = (float)bzero;
    const unsigned grid = (unsigned)std::min<long long>((n + 255) / 256, 148LL * 16);
    const unsigned char *raw = static_cast<const unsigned char *>(d_raw);
    switch (bitpix) {
    case 8: k_fits_to_float<8><<<grid, 256, 0, st>>>(raw, d_out, n, bs, bz, has_blank, blank); return true;
    case 16: k_fits_to_float<16><<<grid, 256, 0, st>>>(raw, d_out, n, bs, bz, has_blank, blank); return true;
    case 32: k_fits_to_float<32><<<grid, 256, 0, st>>>(raw, d_out, n, bs, bz, has_blank, blank); return true;
    case -32: k_fits_to_float<-32><<<grid, 256, 0, st>>>(raw, d_out, n, bs, bz, has_blank, blank); return true;
    case -64: k_fits_to_float<-64><<<grid, 256, 0, st>>>(raw, d_out, n, bs, bz, has_blank, blank); return true;
    }
    return false;
}

}  // namespace sx
