// Internal interface between the C ABI layer (capi.cu) and the kernel files.
// Every launcher enqueues on `st` and returns a cudaError_t (cudaSuccess when
// the launch was accepted); it never synchronises.
#pragma once

#include <cstdint>
#include <vector>
#include <cuda_runtime.h>

#include "vb_common.cuh"

namespace vb {

enum Depth : int { k8U = 0, k16U = 2, k16S = 3, k32S = 4, k32F = 5 };

inline int depth_size(int d) { return d == k8U ? 1 : (d == k16U || d == k16S) ? 2 : (d == k32F || d == k32S) ? 4 : 0; }

// Counts kernel launches made by the library (reported by visar_cuda_launch_count).
void note_launch(int n = 1);
// The calling thread's stream and async flag (visar_cuda_set_stream / _async).
cudaStream_t thread_stream();
int thread_async();
void set_thread_stream(cudaStream_t st, int async);
// Records `msg` as the thread's last error and returns `status`.
int report_error(int status, const char *msg);

// ------------------------------------------------------------- color
// Conversion kinds of src/imgproc/color.zig:44-46.
enum ColorKind : int { kReorder, kGray, kFromGray, kHsv, kFromHsv, kYcrcb, kFromYcrcb };
struct ColorInfo {
  int scn, dcn, sb, db;
  ColorKind kind;
};
cudaError_t launch_cvt_color(const DImg &s, const DImg &d, int depth, const ColorInfo &ci, cudaStream_t st);
// RGB -> gray in 15-bit fixed point (src/imgproc/color.zig:120-130, 8- and 16-bit).
constexpr int kGrayShift = 15, kB2G = 3735, kG2G = 19235, kR2G = 9798;

// ---------------------------------------------------- separable filter
// Finishing step of a separable filter (src/imgproc/filter.zig:60-116).
enum Finish : int {
  kFinShift,   // (v + 2^(s-1)) >> s, clamped to D's maximum (u8 / u16 fixed point)
  kFinCast,    // saturating cast (satV)
  kFinScaled,  // f32(v) * f32(scale), saturating cast
};
// Accumulator kinds: exact integers, or f32 in VISAR's operation order.
enum Acc : int { kAccI32, kAccI64, kAccF32 };

struct SepSpec {
  int sdepth, ddepth;
  Acc acc;
  Finish fin;
  int shift;      // kFinShift
  double scale;   // kFinScaled
  std::vector<int> kxi, kyi;    // integer taps (kAccI32 / kAccI64)
  std::vector<float> kxf, kyf;  // f32 taps (kAccF32)
  int border;
};
cudaError_t launch_sep_filter(const DImg &s, const DImg &d, const SepSpec &spec, cudaStream_t st);
// Register-window kernel for 3x3/5x5/7x7 u8 fixed-point and f32 filters on
// 1/3/4 channels; cudaErrorNotSupported for any other shape. rows_hint <= 0
// picks the row-band height from the image size.
cudaError_t launch_sep_fast(const DImg &s, const DImg &d, const SepSpec &spec, int rows_hint, cudaStream_t st);

// ----------------------------------------------------------- resize
struct alignas(16) LinTap { int o0, o1, w0, w1; };  // u8 bilinear tap (offsets in pixels or rows)
struct CubTap { int o[4]; int w[4]; };            // u8 bicubic tap
struct FLinTap { int o0, o1; float a0, a1; };      // generic bilinear
struct FCubTap { int o[4]; float w[4]; };          // generic bicubic
struct AreaEnt { int di, si; float alpha; };       // INTER_AREA table entry

cudaError_t launch_resize_nearest(const DImg &s, const DImg &d, int depth, const int *xofs_dev, const int *yofs_dev, cudaStream_t st);
cudaError_t launch_resize_u8_linear(const DImg &s, const DImg &d, const LinTap *xt, const LinTap *yt, cudaStream_t st);
cudaError_t launch_resize_u8_half(const DImg &s, const DImg &d, cudaStream_t st);
cudaError_t launch_resize_u8_cubic(const DImg &s, const DImg &d, const CubTap *xt, const CubTap *yt, cudaStream_t st);
cudaError_t launch_resize_area_int(const DImg &s, const DImg &d, int depth, int ix, int iy, bool u8fast, cudaStream_t st);
cudaError_t launch_resize_area_frac(const DImg &s, const DImg &d, int depth, const AreaEnt *xtab, int nx,
                                    const int *xstart, const AreaEnt *ytab, const int *ystart, cudaStream_t st);
cudaError_t launch_resize_linear_generic(const DImg &s, const DImg &d, int depth, const FLinTap *xt, const FLinTap *yt, cudaStream_t st);
cudaError_t launch_resize_cubic_generic(const DImg &s, const DImg &d, int depth, const FCubTap *xt, const FCubTap *yt, cudaStream_t st);
cudaError_t launch_copy_image(const DImg &s, const DImg &d, int depth, cudaStream_t st);

// -------------------------------------------------------------- warps
cudaError_t launch_warp_affine(const DImg &s, const DImg &d, int depth, const float m[6], int interp, int border,
                               double value, cudaStream_t st);
cudaError_t launch_warp_perspective(const DImg &s, const DImg &d, int depth, const double m[9], int interp, int border,
                                    double value, cudaStream_t st);

// ---------------------------------------------------------- threshold
// Applies a fixed threshold. For u8 the LUT decides (covers every type and
// out-of-range threshold); other depths compare.
cudaError_t launch_threshold_lut_u8(const DImg &s, const DImg &d, const uint8_t *lut_dev, cudaStream_t st);
cudaError_t launch_threshold_cmp(const DImg &s, const DImg &d, int depth, int type, double t, double m, cudaStream_t st);
// Auto threshold (Otsu / triangle) of a u8 one-channel image: histogram, then
// the f64 scan on the device; the chosen threshold is written to *thresh_dev
// and the u8 LUT of `type` to lut_dev.
cudaError_t launch_threshold_auto_u8(const DImg &s, int method, int type, double maxval, uint32_t *hist_dev,
                                     double *thresh_dev, uint8_t *lut_dev, cudaStream_t st);
cudaError_t launch_fill(const DImg &d, int depth, double value, cudaStream_t st);

// -------------------------------------------------------- morphology
struct MorphRun { int ky, x0, len; };
cudaError_t launch_morph_pass(const DImg &s, const DImg &d, int depth, bool is_max, int kw, int kh, int ax, int ay,
                              const MorphRun *runs_dev, int nruns, bool rect, cudaStream_t st);
cudaError_t launch_sub_sat(const DImg &a, const DImg &b, const DImg &d, int depth, cudaStream_t st);
// u8 pass for centred-run elements with a horizontal reach <= 4 samples;
// cudaErrorNotSupported otherwise.
cudaError_t launch_morph_fast(const DImg &s, const DImg &d, bool is_max, const std::vector<uint8_t> &mask, int kw, int kh,
                              cudaStream_t st);

// ------------------------------------------------ fused gray + shrink
// grayDownsample (src/videoio/frame.zig:169-335): BGR / BGRA u8 -> gray
// shrunk by the integer factor k (1-16); d is (s.w / k) x (s.h / k).
cudaError_t launch_gray_downsample(const DImg &s, const DImg &d, int k, cudaStream_t st);

// ------------------------------------------------------------ pyramids
// pyrDown (src/imgproc/pyramid.zig:73-96): d is ((w+1)/2, (h+1)/2); any border
// but constant. pyrUp (:408-426): d is (2w, 2h), reflect101 only.
cudaError_t launch_pyr_down(const DImg &s, const DImg &d, int depth, int border, cudaStream_t st);
cudaError_t launch_pyr_up(const DImg &s, const DImg &d, int depth, cudaStream_t st);

// ------------------------------------------------- undistort and remap
// src/calib3d/undistort.zig. Parameter blocks are built on the host into
// byte vectors (one per stripe of undistort's rows, or one for the map) and
// passed as device copies (undistort) or by value (the map).
int undistort_stripe_rows(int width, int height);
// True when the camera of some undistort stripe is singular (its rows are
// then left as they are).
bool undistort_any_singular(const double *new_k, const double K[9], int width, int height);
bool undistort_map_params(const double K[9], const double k8[8], const double *R, const double *new_k,
                          std::vector<uint8_t> &out);
cudaError_t launch_undistort(const DImg &s, const DImg &d, const double K[9], const double k8[8], const double *new_k,
                             cudaStream_t st);
cudaError_t launch_init_undistort_map(const std::vector<uint8_t> &params, const DImg &mx, const DImg &my, cudaStream_t st);
cudaError_t launch_remap(const DImg &s, const DImg &d, const DImg &mx, const DImg &my, uint8_t value, cudaStream_t st);

// ------------------------------------------- tracker tail (tail.cu)
cudaError_t launch_equalize_hist(const DImg &s, const DImg &d, uint32_t *hist_dev, uint8_t *lut_dev, cudaStream_t st);
cudaError_t launch_adaptive_cmp(const DImg &s, const DImg &m, const DImg &d, int idelta, bool inv, uint8_t imax,
                                cudaStream_t st);
cudaError_t launch_convert_u8_f32(const DImg &s, const DImg &d, bool to_f32, cudaStream_t st);
cudaError_t launch_background(const DImg &f, const DImg &m, uint16_t *model, int t, int shift, bool primed, cudaStream_t st);
// Connected components: device work buffers (P, K: one int per pixel; F, R:
// one u32 per key; tmp: cc_scan_tmp_words(keys) u32; err, total: one each).
struct CcBuffers {
  int *P, *K;
  uint32_t *F, *R, *tmp;
  int *err;
  uint32_t *total;
};
size_t cc_scan_tmp_words(long long n);
size_t cc_acc_bytes();
// Labels by union-find, keys, ranks; *total receives the component count.
cudaError_t launch_cc_phase1(const DImg &s, bool eight, const CcBuffers &b, cudaStream_t st);
// The label image and per-label accumulators (nlabels = components + 1).
cudaError_t launch_cc_phase2(const DImg &labels, bool eight, const CcBuffers &b, void *acc, int nlabels, cudaStream_t st);
// x0, y0, x1, y1, area, twice the x sum, y sum of accumulator i (host copy).
void cc_read_acc(const void *host_acc, int i, long long out[7]);

// ------------------------------------------------------- host helpers
// Gaussian taps (src/imgproc/filter.zig:350-476), in host f64.
void gaussian_kernel(double *out, int n, double sigma);
int gaussian_ksize(double sigma, bool depth_is_u8);
void gaussian_kernel_fixed(int64_t *out, int n, double sigma, int bits);
// getDerivKernels (src/imgproc/filter.zig:817-854). Returns false for an invalid kernel.
bool deriv_kernel(int *out, int n, int order, int ksize);
// sat.cast(i16, f32).
int sat_i16(float x);
// linearTapU8 (src/imgproc/resize.zig:181-214) for destination index d.
LinTap lin_tap_u8(long long d, uint32_t ssize, uint32_t dsize, bool area, bool pin);
// linearCoord + Weights(T).coef (src/imgproc/resize.zig:156-179, 410-415): generic bilinear taps.
FLinTap lin_tap_f(long long d, uint32_t ssize, uint32_t dsize, bool area, bool is_x);
// getStructuringElement (src/imgproc/morph.zig:32-59): h x w mask, row-major.
std::vector<uint8_t> structuring_element(int shape, int w, int h);
// warpAffine's inverse map in f32 / warpPerspective's in f64; false if singular.
bool affine_inverse_f32(const double m[6], float out[6]);
bool perspective_inverse(const double m[9], double out[9]);

// ------------------------------------- resize with a static tap buffer
// Largest destination width or height of the allocation-free linear resize.
constexpr int kNoAllocMaxSide = 16384;
cudaError_t static_taps_on_device(int dev, LinTap **out);
cudaError_t launch_resize_linear_u8_static(const DImg &s, const DImg &d, LinTap *taps, cudaStream_t st);

}  // namespace vb
