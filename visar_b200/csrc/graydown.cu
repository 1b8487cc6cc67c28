// Fused BT.601 gray + integer box shrink of a BGR / BGRA u8 image
// (grayDownsample, src/videoio/frame.zig:169-335): no full-size gray image is
// written; every source byte is read once.
//
// Arithmetic (frame.zig:190-193, 287-335). With s_b, s_g, s_r the k x k block
// sums of the B, G and R samples and l = s_b*1868 + s_g*9617 + s_r*4899 (u32):
//   k == 2: (l + 2^15) >> 16                                    (`pairs`)
//   else:   trunc(min(255, f32(l) * f32(1 / (k*k*2^14)) + 0.5)) (`blocks`)
// each f32 operation rounded on its own (the library is built without
// contraction, so the multiply and the add stay separate).
//
// Layout: a CTA owns one output row and a chunk of P output pixels (P a
// multiple of 16, P*k*cn <= 4096 source bytes per row). Phase 1: each thread
// sums the k source rows of 16-byte columns of the chunk (16-bit lanes, two
// per register) and writes the per-byte sums to shared memory. Phase 2: each
// thread reduces k*cn consecutive sums per output pixel and stores it.
#include "vb.h"

namespace vb {
namespace {

constexpr uint32_t kWb = 1868, kWg = 9617, kWr = 4899;
constexpr int kChunkBytes = 4096;
constexpr int kThreads = 128;

__device__ __forceinline__ void add_bytes(uint32_t w, uint32_t &lo, uint32_t &hi) {
  lo += __byte_perm(w, 0, 0x4140);  // bytes 0, 1 as 16-bit lanes
  hi += __byte_perm(w, 0, 0x4342);  // bytes 2, 3
}

template <int CN>
__global__ void __launch_bounds__(kThreads) k_gray_down(const uint8_t *__restrict__ src, long long sstride,
                                                        uint8_t *__restrict__ dst, long long dstride, int dw, int dh,
                                                        int k, int P, float inv, bool vec_ok) {
  __shared__ __align__(16) uint16_t sums[kChunkBytes];
  const int px0 = blockIdx.x * P;
  const int npx = min(P, dw - px0);
  const long long used = (long long)npx * k * CN;  // source bytes of this chunk per row
  const long long off0 = (long long)px0 * k * CN;
  const int nvec = (int)((used + 15) >> 4);
  for (int oy = blockIdx.y; oy < dh; oy += gridDim.y) {
    const uint8_t *row0 = src + (long long)oy * k * sstride + off0;
    for (int v = threadIdx.x; v < nvec; v += kThreads) {
      uint32_t acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      const long long b = (long long)v * 16;
      if (vec_ok && b + 16 <= used) {
        const uint8_t *p = row0 + b;
#pragma unroll 4
        for (int r = 0; r < k; r++, p += sstride) {
          const uint4 q = __ldg(reinterpret_cast<const uint4 *>(p));
          add_bytes(q.x, acc[0], acc[1]);
          add_bytes(q.y, acc[2], acc[3]);
          add_bytes(q.z, acc[4], acc[5]);
          add_bytes(q.w, acc[6], acc[7]);
        }
      } else {
        const int n = (int)min(16LL, used - b);
        const uint8_t *p = row0 + b;
        for (int r = 0; r < k; r++, p += sstride)
          for (int i = 0; i < n; i++) acc[i >> 1] += (uint32_t)p[i] << ((i & 1) * 16);
      }
      uint4 *o = reinterpret_cast<uint4 *>(sums + b);
      o[0] = make_uint4(acc[0], acc[1], acc[2], acc[3]);
      o[1] = make_uint4(acc[4], acc[5], acc[6], acc[7]);
    }
    __syncthreads();
    uint8_t *drow = dst + (long long)oy * dstride + px0;
    for (int j = threadIdx.x; j < npx; j += kThreads) {
      const uint16_t *s = sums + j * k * CN;
      uint32_t sb = 0, sg = 0, sr = 0;
      for (int i = 0; i < k; i++, s += CN) {
        sb += s[0];
        sg += s[1];
        sr += s[2];
      }
      const uint32_t l = sb * kWb + sg * kWg + sr * kWr;
      uint32_t out;
      if (k == 2) {
        out = (l + (1u << 15)) >> 16;
      } else {
        const float f = fminf(255.0f, __fadd_rn(__fmul_rn(__uint2float_rn(l), inv), 0.5f));
        out = (uint32_t)f;
      }
      drow[j] = (uint8_t)out;
    }
    __syncthreads();
  }
}

}  // namespace

int gray_down_chunk(int k, int cn) {
  int p = kChunkBytes / (k * cn);
  p -= p % 16;
  return p < 16 ? 16 : p;
}

cudaError_t launch_gray_downsample(const DImg &s, const DImg &d, int k, cudaStream_t st) {
  const int P = gray_down_chunk(k, s.cn);
  if ((long long)P * k * s.cn > kChunkBytes) return cudaErrorInvalidValue;
  const float inv = 1.0f / (float)(k * k * (1 << 14));
  const bool vec_ok = ((uintptr_t)s.p % 16 == 0) && (s.stride % 16 == 0);
  dim3 grid((d.w + P - 1) / P, (unsigned)min(d.h, 65535));
  note_launch();
  if (s.cn == 4)
    k_gray_down<4><<<grid, kThreads, 0, st>>>(s.p, s.stride, d.p, d.stride, d.w, d.h, k, P, inv, vec_ok);
  else
    k_gray_down<3><<<grid, kThreads, 0, st>>>(s.p, s.stride, d.p, d.stride, d.w, d.h, k, P, inv, vec_ok);
  return cudaGetLastError();
}

}  // namespace vb
