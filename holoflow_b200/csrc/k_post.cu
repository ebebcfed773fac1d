// Post-moment display chain: the steps Holoflow applies to a moment image before it is shown
// (graph_builder.cc:633-676): fftshift, flatfield (Gaussian high-pass), sliding average over
// pp_accumulation images, percentile clip inside an elliptical region, then the Scaled U8
// conversion (hf_convert, k_misc.cu).  All are memory-bound passes over one image per window.
//
//  - hf_fftshift follows holonp/src/fftshift.cu:98-134: out[j] = in[(j + n/2) mod n] on each
//    shifted axis (numpy's fftshift for even n; for odd n this is the reference's own choice).
//  - hf_flatfield follows holotask/src/syncs/flatfield.cu: out = in - G * in.  Kernels shorter
//    than 65 taps run the separable Gaussian in shared-memory tiles with clamp-at-edge borders
//    (the taps built on the host exactly as make_gaussian_kernel, lines 57-77, and summed in the
//    same order); longer ones take the analytic Fourier high-pass
//    (1 - exp(-2 pi^2 (sx^2 fx^2 + sy^2 fy^2))) / (W H) through this library's own four-step
//    row / column passes.  The reference writes sigma and 1 / (W H) into a JIT source with
//    std::to_string (six decimals, flatfield.cu:124-131); the same rounding is applied here so
//    that the two agree (for a 1024 x 1024 image 1 / (W H) becomes 1e-6, a 4.9 % larger gain; the
//    later Scaled conversion to U8 removes any global gain).
//  - hf_slideavg follows holotask/src/asyncs/slide_avg.cu:211-250: a running average kept as
//    avg += x / n, avg -= x_(k-n) / n in float32 in that order, the ring starting at zero, and an
//    image out once n images (after discard_first) have gone in.
//  - hf_pctclip follows holotask/src/syncs/pct_clip.cu: the values at ranks
//    int(p / 100 (count - 1)) of the pixels inside the ellipse (all slices), then
//    min(max(x, lo), hi) on every pixel.  Instead of a full radix sort, an exact radix select:
//    four passes of 8-bit shared-memory histograms over the same order-preserving float key
//    (sign bit set for positives, all bits inverted for negatives) find both ranks at once.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "hf_common.cuh"
#include "k_fft2d.cuh"
#include "k_post.cuh"

namespace hf {
namespace {

// ------------------------------------------------------------------------------------------------
// fftshift
// ------------------------------------------------------------------------------------------------
constexpr int kShiftMaxDim = 16;
struct ShiftGeom {
  int     ndim;
  int64_t shape[kShiftMaxDim], stride[kShiftMaxDim], shift[kShiftMaxDim]; // strides in elements
};

template <typename E>
__global__ void fftshift_kernel(const E *__restrict__ in, E *__restrict__ out, ShiftGeom g, int64_t total) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    int64_t rem = i, src = 0;
    for (int k = 0; k < g.ndim; ++k) {
      const int64_t o = rem / g.stride[k];
      rem -= o * g.stride[k];
      int64_t s = o + g.shift[k];
      if (s >= g.shape[k])
        s -= g.shape[k];
      src += s * g.stride[k];
    }
    out[i] = in[src];
  }
}
struct Bytes3 {
  uint8_t b[3];
};
struct Bytes16 {
  uint4 v;
};

// ------------------------------------------------------------------------------------------------
// flatfield, spatial path
// ------------------------------------------------------------------------------------------------
constexpr int kFfMaxRadius = 31; // kernels of up to 63 taps; 65 and longer take the Fourier path
struct Taps {
  int   r;
  float w[2 * kFfMaxRadius + 1];
};
constexpr int kFfRowTile = 256;
constexpr int kFfColTile = 64; // output rows per vertical tile (32 columns, 8 warps x 8 rows)

// temp = horizontal Gaussian of each row (clamped at the row ends)
__global__ void __launch_bounds__(kFfRowTile) flatfield_rows_kernel(const float *__restrict__ in,
                                                                    float *__restrict__ tmp, int H, int W,
                                                                    Taps t) {
  __shared__ float tile[kFfRowTile + 2 * kFfMaxRadius];
  const int64_t plane = (int64_t)blockIdx.z * H * W;
  const int     y = blockIdx.y, x0 = blockIdx.x * kFfRowTile;
  const float  *row = in + plane + (int64_t)y * W;
  for (int j = threadIdx.x; j < kFfRowTile + 2 * t.r; j += blockDim.x) {
    const int x = min(max(x0 - t.r + j, 0), W - 1);
    tile[j]     = row[x];
  }
  __syncthreads();
  const int x = x0 + threadIdx.x;
  if (x >= W)
    return;
  float sum = 0.f;
  for (int k = 0; k <= 2 * t.r; ++k)
    sum = fmaf(tile[threadIdx.x + k], t.w[k], sum);
  tmp[plane + (int64_t)y * W + x] = sum;
}

// out = in - vertical Gaussian of temp (clamped at the column ends)
__global__ void __launch_bounds__(256) flatfield_cols_kernel(const float *__restrict__ in,
                                                             const float *__restrict__ tmp,
                                                             float *__restrict__ out, int H, int W, Taps t) {
  __shared__ float tile[kFfColTile + 2 * kFfMaxRadius][32];
  const int64_t plane = (int64_t)blockIdx.z * H * W;
  const int     x = blockIdx.x * 32 + threadIdx.x, y0 = blockIdx.y * kFfColTile;
  const int     xc = min(x, W - 1);
  for (int j = threadIdx.y; j < kFfColTile + 2 * t.r; j += blockDim.y) {
    const int y      = min(max(y0 - t.r + j, 0), H - 1);
    tile[j][threadIdx.x] = tmp[plane + (int64_t)y * W + xc];
  }
  __syncthreads();
  if (x >= W)
    return;
  for (int m = threadIdx.y; m < kFfColTile; m += blockDim.y) {
    const int y = y0 + m;
    if (y >= H)
      break;
    float bg = 0.f;
    for (int k = 0; k <= 2 * t.r; ++k)
      bg = fmaf(tile[m + k][threadIdx.x], t.w[k], bg);
    const int64_t i = plane + (int64_t)y * W + x;
    out[i]          = in[i] - bg;
  }
}

// ------------------------------------------------------------------------------------------------
// flatfield, Fourier path helpers
// ------------------------------------------------------------------------------------------------
__global__ void flatfield_gain_kernel(float2 *gain, int H, int W, float sy, float sx, float scale) {
  const int64_t n = (int64_t)H * W;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int   y = (int)(i / W), x = (int)(i % W);
    // the full spectrum's column x stands for frequency x or x - W; the gain depends on fx^2
    const int   xf = x <= W / 2 ? x : W - x;
    const float fx = (float)xf / (float)W;
    const float fy = (float)(y <= H / 2 ? y : y - H) / (float)H;
    constexpr float two_pi_squared = 19.739208802178716f;
    const float lowpass = expf(-two_pi_squared * (sx * sx * fx * fx + sy * sy * fy * fy));
    gain[i]             = make_float2((1.0f - lowpass) * scale, 0.f);
  }
}

__global__ void real_part_kernel(const float2 *__restrict__ c, float *__restrict__ out, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = c[i].x;
}

// ------------------------------------------------------------------------------------------------
// filter2d (holotask/src/syncs/filter2d.cu:109-199): the band-pass annulus a (1 - b) in the
// transform's natural frequency order.  Complex input: the reference builds the centred mask,
// swaps its corners (fftshift for even sides) and stores (g, g) -- a complex factor sqrt(2)
// e^(i pi / 4) that is kept here.  Real input: the R2C half spectrum's (g, 0) with the
// `smooth > 0` guards, extended to the full spectrum by the symmetry of |f|.
// ------------------------------------------------------------------------------------------------
__device__ float annulus(float dist, float ri, float ro, float si, float so, bool guards) {
  float a = 0.0f, b = 0.0f;
  if (dist < ro)
    a = 1.0f;
  else if ((!guards || so > 0.0f) && dist < ro + so)
    a = cosf((dist - ro) / so * 3.14159265358979323846f / 2);
  if (dist < ri)
    b = 1.0f;
  else if ((!guards || si > 0.0f) && dist < ri + si)
    b = cosf((dist - ri) / si * 3.14159265358979323846f / 2);
  return a * (1 - b);
}

__global__ void filter2d_table_kernel(float2 *tab, int W, int H, uint32_t ri, uint32_t ro, uint32_t si, uint32_t so,
                                      int real_in) {
  const int64_t n = (int64_t)H * W;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int y = (int)(i / W), x = (int)(i % W);
    float     g;
    if (real_in) {
      const int   xf = x <= W / 2 ? x : W - x;
      const int   fy = y <= H / 2 ? y : y - H;
      const float dist = hypotf((float)xf, (float)fy);
      g                = annulus(dist, (float)ri, (float)ro, (float)si, (float)so, true);
      tab[i]           = make_float2(g, 0.f);
    } else {
      const int   xc = (x + W / 2) % W, yc = (y + H / 2) % H; // the centred mask's pixel here
      const float rx = (float)xc - (float)W / 2, ry = (float)yc - (float)H / 2;
      g              = annulus(hypotf(rx, ry), (float)ri, (float)ro, (float)si, (float)so, false);
      tab[i]         = make_float2(g, g);
    }
  }
}

// ------------------------------------------------------------------------------------------------
// percentile clip
// ------------------------------------------------------------------------------------------------
struct SelState {
  uint32_t prefix[2], rank[2];
  uint32_t hist[2][256];
  float    lo, hi;
};

__device__ __forceinline__ uint32_t float_key(float v) {
  const uint32_t u = __float_as_uint(v);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float key_float(uint32_t k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k);
}

__device__ bool in_ellipse(int x, int y, int width, int height, float cx, float cy, float rx, float ry, float angle) {
  if (width <= 0 || height <= 0 || rx <= 0.f || ry <= 0.f)
    return false;
  const float xn = ((float)x + 0.5f) / (float)width;
  const float yn = ((float)y + 0.5f) / (float)height;
  const float dx = xn - cx, dy = yn - cy;
  const float th = angle * (3.14159265358979323846f / 180.0f);
  const float c = cosf(th), s = sinf(th);
  const float xr = c * dx + s * dy;
  const float yr = -s * dx + c * dy;
  return (xr * xr) / (rx * rx) + (yr * yr) / (ry * ry) <= 1.0f;
}

__global__ void roi_mask_kernel(uint8_t *mask, int *count, int W, int H, int D, float cx, float cy, float rx,
                                float ry, float angle) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y, z = blockIdx.z;
  if (x >= W || y >= H || z >= D)
    return;
  const bool sel = in_ellipse(x, y, W, H, cx, cy, rx, ry, angle);
  mask[((int64_t)z * H + y) * W + x] = sel;
  if (sel)
    atomicAdd(count, 1);
}

__global__ void select_init_kernel(SelState *st, uint32_t rank_lo, uint32_t rank_hi) {
  for (int i = threadIdx.x; i < 512; i += blockDim.x)
    (&st->hist[0][0])[i] = 0u;
  if (threadIdx.x == 0) {
    st->prefix[0] = st->prefix[1] = 0u;
    st->rank[0] = rank_lo, st->rank[1] = rank_hi;
  }
}

__global__ void __launch_bounds__(256) select_hist_kernel(const float *__restrict__ in, const uint8_t *__restrict__ mask,
                                                          int64_t n, SelState *st, int pass) {
  __shared__ uint32_t h[2][256];
  for (int i = threadIdx.x; i < 512; i += blockDim.x)
    (&h[0][0])[i] = 0u;
  __syncthreads();
  const int      shift   = 24 - 8 * pass;
  const uint32_t hi_mask = pass == 0 ? 0u : (0xFFFFFFFFu << (shift + 8));
  const uint32_t p0 = st->prefix[0] & hi_mask, p1 = st->prefix[1] & hi_mask;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (!mask[i])
      continue;
    const uint32_t k   = float_key(in[i]);
    const uint32_t bin = (k >> shift) & 255u;
    if ((k & hi_mask) == p0)
      atomicAdd(&h[0][bin], 1u);
    if ((k & hi_mask) == p1)
      atomicAdd(&h[1][bin], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 512; i += blockDim.x) {
    const uint32_t c = (&h[0][0])[i];
    if (c)
      atomicAdd(&(&st->hist[0][0])[i], c);
  }
}

__global__ void select_step_kernel(SelState *st, int pass) {
  const int shift = 24 - 8 * pass;
  if (threadIdx.x < 2) {
    const int t   = threadIdx.x;
    uint32_t  cum = 0, bin = 255;
    for (uint32_t b = 0; b < 256; ++b) {
      const uint32_t c = st->hist[t][b];
      if (cum + c > st->rank[t]) {
        bin = b;
        break;
      }
      cum += c;
    }
    st->rank[t] -= cum;
    st->prefix[t] |= bin << shift;
    if (pass == 3) {
      if (t == 0)
        st->lo = key_float(st->prefix[0]);
      else
        st->hi = key_float(st->prefix[1]);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 512; i += blockDim.x)
    (&st->hist[0][0])[i] = 0u;
}

__global__ void clip_kernel(const float *__restrict__ in, float *__restrict__ out, int64_t n, const SelState *st) {
  const float lo = st->lo, hi = st->hi;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = fminf(fmaxf(in[i], lo), hi);
}

// ------------------------------------------------------------------------------------------------
// sliding average
// ------------------------------------------------------------------------------------------------
__global__ void slideavg_kernel(const float *__restrict__ x, float *__restrict__ slot, float *__restrict__ avg,
                                float *__restrict__ out, int64_t n, float window) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float xi = x[i], old = slot[i];
    float       a  = avg[i] + __fdiv_rn(xi, window);
    a              = a - __fdiv_rn(old, window);
    avg[i]         = a;
    slot[i]        = xi;
    if (out)
      out[i] = a;
  }
}

int grid_for(int64_t n, int block = 256) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((n + block - 1) / block, (int64_t)sm_count() * 16));
}

// std::to_string(float) keeps six decimals: the value the reference's JIT source compiles in
float six_decimals(float v) { return std::stof(std::to_string(v)); }

} // namespace

// out = IFFT2(FFT2(in) x tab) per [H][W] plane, unnormalized both ways (as the reference's cuFFT
// pair): rows forward into the scratch spectrum c0, the columns' transfer-function sandwich with
// the mask in place, rows inverse into `out` (complex) or into c1 and its real part (real).
int launch_filter2d(const float2 *tab, int64_t planes, int H, int W, int real_in, const void *in, void *out,
                    float2 *c0, float2 *c1, cudaStream_t s) {
  const int64_t P = (int64_t)H * W;
  RowPass       rp{};
  rp.in = in, rp.in_real = real_in, rp.in_win = planes * P, rp.in_plane = P, rp.in_row = W, rp.in_col = 1;
  rp.IH = H, rp.IW = W, rp.oy = 0, rp.ox = 0, rp.H = H, rp.N = W, rp.nplanes = (int)planes, rp.inverse = 0;
  rp.out = c0, rp.out_win = planes * P, rp.out_plane = P, rp.out_row = W;
  HF_TRY(launch_row_pass(rp, 1, s));
  ColPass cp{};
  cp.in = c0, cp.in_win = planes * P, cp.in_plane = P, cp.in_row = W, cp.H = H, cp.W = W, cp.nplanes = (int)planes;
  cp.out = c0, cp.out_win = planes * P, cp.out_plane = P, cp.out_row = W, cp.out_col = 1, cp.tf = tab, cp.inverse = 0;
  HF_TRY(launch_col_pass(cp, COL_TF_SANDWICH, nullptr, 1, s));
  RowPass ri = rp;
  ri.in = c0, ri.in_real = 0, ri.inverse = 1;
  ri.out = real_in ? c1 : static_cast<float2 *>(out);
  HF_TRY(launch_row_pass(ri, 1, s));
  if (!real_in)
    return HF_OK;
  real_part_kernel<<<grid_for(planes * P), 256, 0, s>>>(c1, static_cast<float *>(out), planes * P);
  note_launch();
  return launch_status("real_part_kernel");
}

// The annulus mask in natural frequency order for a complex (real_in = 0) or real input.
int launch_filter2d_table(float2 *tab, int H, int W, int real_in, uint32_t ri, uint32_t ro, uint32_t si, uint32_t so,
                          cudaStream_t s) {
  filter2d_table_kernel<<<grid_for((int64_t)H * W), 256, 0, s>>>(tab, W, H, ri, ro, si, so, real_in);
  note_launch();
  return launch_status("filter2d_table_kernel");
}

} // namespace hf

using namespace hf;

struct hf_flatfield {
  int64_t planes = 0;
  int     H = 0, W = 0;
  bool    fourier = false;
  Taps    ty{}, tx{};
  float  *tmp  = nullptr; // spatial: horizontal pass
  float2 *gain = nullptr; // Fourier: [H][W] gain
  float2 *c0 = nullptr, *c1 = nullptr;
};

struct hf_filter2d {
  int64_t planes = 0;
  int     H = 0, W = 0, real_in = 0;
  float2 *tab = nullptr, *c0 = nullptr, *c1 = nullptr;
};

struct hf_pctclip {
  int      D = 0, H = 0, W = 0;
  int      count = 0, min_idx = 0, max_idx = 0;
  uint8_t *mask = nullptr;
  SelState *st  = nullptr;
};

struct hf_slideavg {
  int64_t npix = 0;
  int     window = 0, discard_first = 0, discarded = 0, slot = 0;
  int64_t pushes = 0;
  float  *ring = nullptr, *avg = nullptr;
};

namespace {
// Releases without touching the error message (create's failure paths keep their reason).
void release(hf_flatfield *f) {
  if (f) {
    cudaFree(f->tmp);
    cudaFree(f->gain);
    cudaFree(f->c0);
    cudaFree(f->c1);
    delete f;
  }
}
void release(hf_filter2d *f) {
  if (f) {
    cudaFree(f->tab);
    cudaFree(f->c0);
    cudaFree(f->c1);
    delete f;
  }
}
void release(hf_pctclip *p) {
  if (p) {
    cudaFree(p->mask);
    cudaFree(p->st);
    delete p;
  }
}
void release(hf_slideavg *a) {
  if (a) {
    cudaFree(a->ring);
    cudaFree(a->avg);
    delete a;
  }
}

// make_gaussian_kernel (flatfield.cu:57-77): radius ceil(3 sigma), exp in float, normalised by
// the float sum accumulated in tap order.
bool gaussian_taps(float sigma, std::vector<float> &w) {
  const int radius = (int)std::ceil(3.0f * sigma);
  if (radius <= 0)
    return false;
  w.assign((size_t)(2 * radius + 1), 0.f);
  const float inv_two_sigma2 = 1.0f / (2.0f * sigma * sigma);
  float       sum            = 0.0f;
  for (int i = -radius; i <= radius; ++i) {
    const float v       = std::exp(-(float)(i * i) * inv_two_sigma2);
    w[(size_t)(i + radius)] = v;
    sum += v;
  }
  for (auto &v : w)
    v /= sum;
  return true;
}
} // namespace

extern "C" {

int hf_fftshift(const void *in, void *out, int elem_size, int ndim, const int64_t *shape, uint32_t axes_mask,
                hf_stream_t s) {
  clear_error();
  HF_CHECK_ARG(in != nullptr && out != nullptr && shape != nullptr, "FFTShift: null argument");
  HF_CHECK_ARG(in != out, "FFTShift: input and output must not alias");
  HF_CHECK_ARG(ndim > 0 && ndim <= kShiftMaxDim, "FFTShift: input ndim must be in [1, 16]");
  HF_CHECK_ARG(elem_size == 1 || elem_size == 2 || elem_size == 3 || elem_size == 4 || elem_size == 8 ||
                   elem_size == 16,
               "FFTShift: element size must be 1, 2, 3, 4, 8 or 16 bytes");
  ShiftGeom g{};
  g.ndim        = ndim;
  int64_t total = 1;
  for (int k = ndim - 1; k >= 0; --k) {
    HF_CHECK_ARG(shape[k] > 0, "FFTShift: input tensor has zero elements");
    g.shape[k]  = shape[k];
    g.stride[k] = total;
    g.shift[k]  = (axes_mask >> k) & 1u ? shape[k] / 2 : 0;
    total *= shape[k];
  }
  const int grid = grid_for(total);
  switch (elem_size) {
  case 1: fftshift_kernel<uint8_t><<<grid, 256, 0, s>>>((const uint8_t *)in, (uint8_t *)out, g, total); break;
  case 2: fftshift_kernel<uint16_t><<<grid, 256, 0, s>>>((const uint16_t *)in, (uint16_t *)out, g, total); break;
  case 3: fftshift_kernel<Bytes3><<<grid, 256, 0, s>>>((const Bytes3 *)in, (Bytes3 *)out, g, total); break;
  case 4: fftshift_kernel<uint32_t><<<grid, 256, 0, s>>>((const uint32_t *)in, (uint32_t *)out, g, total); break;
  case 8: fftshift_kernel<uint2><<<grid, 256, 0, s>>>((const uint2 *)in, (uint2 *)out, g, total); break;
  default: fftshift_kernel<Bytes16><<<grid, 256, 0, s>>>((const Bytes16 *)in, (Bytes16 *)out, g, total); break;
  }
  note_launch();
  return launch_status("fftshift_kernel");
}

int hf_flatfield_create(int64_t planes, int height, int width, float sigma_y, float sigma_x, hf_stream_t s,
                        hf_flatfield **out) {
  clear_error();
  HF_CHECK_ARG(out != nullptr, "Flatfield: null argument");
  *out = nullptr;
  HF_CHECK_ARG(planes >= 1 && height >= 1 && width >= 1, "Flatfield: input must not be empty");
  HF_CHECK_ARG(sigma_y > 0.f, "Flatfield: sigma_y must be positive");
  HF_CHECK_ARG(sigma_x > 0.f, "Flatfield: sigma_x must be positive");
  std::vector<float> ky, kx;
  HF_CHECK_ARG(gaussian_taps(sigma_y, ky) && gaussian_taps(sigma_x, kx),
               "Flatfield: sigma is too small to form a Gaussian kernel");
  // should_use_fft_flatfield (flatfield.cu:169-174)
  const bool fourier = height > 1 && width > 1 && std::max(ky.size(), kx.size()) >= 65;
  auto      *f       = new (std::nothrow) hf_flatfield();
  if (!f)
    return fail(HF_ERR_NOMEM, "Flatfield: host allocation failed");
  f->planes = planes, f->H = height, f->W = width, f->fourier = fourier;
  const size_t npx = (size_t)planes * height * width;
  auto         bad = [&](int rc) {
    release(f);
    return rc;
  };
  if (!fourier) {
    if (std::max(ky.size(), kx.size()) > 2 * kFfMaxRadius + 1)
      return bad(fail(HF_ERR_UNSUPPORTED, "Flatfield: a kernel of 65 or more taps on a one-pixel-wide image"));
    f->ty.r = (int)ky.size() / 2, f->tx.r = (int)kx.size() / 2;
    std::memcpy(f->ty.w, ky.data(), ky.size() * sizeof(float));
    std::memcpy(f->tx.w, kx.data(), kx.size() * sizeof(float));
    const int rc = cuda_status(cudaMalloc(&f->tmp, npx * sizeof(float)), "Flatfield: temporary");
    if (rc != HF_OK)
      return bad(rc);
  } else {
    if (!(fft_fast_length(height) && fft_fast_length(width) && height <= 1024))
      return bad(fail(HF_ERR_UNSUPPORTED, "Flatfield: the Fourier high-pass needs image sides in "
                                          "{64, 128, 256, 512, 768, 1024, 1536} (height <= 1024)"));
    int rc = cuda_status(cudaMalloc(&f->gain, (size_t)height * width * sizeof(float2)), "Flatfield: gain");
    if (rc == HF_OK)
      rc = cuda_status(cudaMalloc(&f->c0, npx * sizeof(float2)), "Flatfield: spectrum");
    if (rc == HF_OK)
      rc = cuda_status(cudaMalloc(&f->c1, npx * sizeof(float2)), "Flatfield: spectrum");
    if (rc != HF_OK)
      return bad(rc);
    const float scale = six_decimals(1.0f / (float)(width * height));
    flatfield_gain_kernel<<<grid_for((int64_t)height * width), 256, 0, s>>>(
        f->gain, height, width, six_decimals(sigma_y), six_decimals(sigma_x), scale);
    note_launch();
    rc = launch_status("flatfield_gain_kernel");
    if (rc != HF_OK)
      return bad(rc);
  }
  *out = f;
  return HF_OK;
}

int hf_flatfield_is_fourier(const hf_flatfield *f, int *fourier) {
  clear_error();
  HF_CHECK_ARG(f != nullptr && fourier != nullptr, "Flatfield: null argument");
  *fourier = f->fourier ? 1 : 0;
  return HF_OK;
}

int hf_flatfield_exec(hf_flatfield *f, const float *in, float *out, hf_stream_t s) {
  clear_error();
  HF_CHECK_ARG(f != nullptr && in != nullptr && out != nullptr, "Flatfield: null argument");
  const int     H = f->H, W = f->W;
  const int64_t P = (int64_t)H * W;
  if (!f->fourier) {
    HF_CHECK_ARG(f->planes <= 65535, "Flatfield: at most 65535 planes");
    flatfield_rows_kernel<<<dim3((W + kFfRowTile - 1) / kFfRowTile, H, (unsigned)f->planes), kFfRowTile, 0, s>>>(
        in, f->tmp, H, W, f->tx);
    note_launch();
    HF_TRY(launch_status("flatfield_rows_kernel"));
    flatfield_cols_kernel<<<dim3((W + 31) / 32, (H + kFfColTile - 1) / kFfColTile, (unsigned)f->planes), dim3(32, 8),
                            0, s>>>(in, f->tmp, out, H, W, f->ty);
    note_launch();
    return launch_status("flatfield_cols_kernel");
  }
  // rows forward (real in) -> columns forward x gain x inverse -> rows inverse -> real part
  RowPass rp{};
  rp.in = in, rp.in_real = 1, rp.in_win = f->planes * P, rp.in_plane = P, rp.in_row = W, rp.in_col = 1;
  rp.IH = H, rp.IW = W, rp.oy = 0, rp.ox = 0, rp.H = H, rp.N = W, rp.nplanes = (int)f->planes, rp.inverse = 0;
  rp.out = f->c0, rp.out_win = f->planes * P, rp.out_plane = P, rp.out_row = W;
  HF_TRY(launch_row_pass(rp, 1, s));
  ColPass cp{};
  cp.in = f->c0, cp.in_win = f->planes * P, cp.in_plane = P, cp.in_row = W, cp.H = H, cp.W = W;
  cp.nplanes = (int)f->planes, cp.out = f->c0, cp.out_win = f->planes * P, cp.out_plane = P, cp.out_row = W;
  cp.out_col = 1, cp.tf = f->gain, cp.inverse = 0;
  HF_TRY(launch_col_pass(cp, COL_TF_SANDWICH, nullptr, 1, s));
  RowPass ri = rp;
  ri.in = f->c0, ri.in_real = 0, ri.out = f->c1, ri.inverse = 1;
  HF_TRY(launch_row_pass(ri, 1, s));
  real_part_kernel<<<grid_for(f->planes * P), 256, 0, s>>>(f->c1, out, f->planes * P);
  note_launch();
  return launch_status("real_part_kernel");
}

int hf_flatfield_destroy(hf_flatfield *f) {
  clear_error();
  release(f);
  return HF_OK;
}

int hf_filter2d_create(int64_t planes, int height, int width, int real_input, uint32_t r_inner, uint32_t r_outer,
                       uint32_t s_inner, uint32_t s_outer, hf_stream_t s, hf_filter2d **out) {
  clear_error();
  HF_CHECK_ARG(out != nullptr, "Filter2D: null argument");
  *out = nullptr;
  HF_CHECK_ARG(planes >= 1 && height >= 1 && width >= 1, "Filter2D: input must not be empty");
  if (!(fft_fast_length(height) && fft_fast_length(width) && height <= 1024))
    return fail(HF_ERR_UNSUPPORTED,
                "Filter2D: image sides must be in {64, 128, 256, 512, 768, 1024, 1536} (height <= 1024)");
  auto *f = new (std::nothrow) hf_filter2d();
  if (!f)
    return fail(HF_ERR_NOMEM, "Filter2D: host allocation failed");
  f->planes = planes, f->H = height, f->W = width, f->real_in = real_input ? 1 : 0;
  const size_t npx = (size_t)planes * height * width;
  int          rc  = cuda_status(cudaMalloc(&f->tab, (size_t)height * width * sizeof(float2)), "Filter2D: mask");
  if (rc == HF_OK)
    rc = cuda_status(cudaMalloc(&f->c0, npx * sizeof(float2)), "Filter2D: spectrum");
  if (rc == HF_OK && real_input)
    rc = cuda_status(cudaMalloc(&f->c1, npx * sizeof(float2)), "Filter2D: spectrum");
  if (rc == HF_OK)
    rc = launch_filter2d_table(f->tab, height, width, f->real_in, r_inner, r_outer, s_inner, s_outer, s);
  if (rc != HF_OK) {
    release(f);
    return rc;
  }
  *out = f;
  return HF_OK;
}

int hf_filter2d_exec(hf_filter2d *f, const void *in, void *out, hf_stream_t s) {
  clear_error();
  HF_CHECK_ARG(f != nullptr && in != nullptr && out != nullptr, "Filter2D: null argument");
  return launch_filter2d(f->tab, f->planes, f->H, f->W, f->real_in, in, out, f->c0, f->c1, s);
}

int hf_filter2d_destroy(hf_filter2d *f) {
  clear_error();
  release(f);
  return HF_OK;
}

int hf_pctclip_create(int depth, int height, int width, float min_pct, float max_pct, const hf_ellipse *roi,
                      hf_stream_t s, hf_pctclip **out) {
  clear_error();
  HF_CHECK_ARG(out != nullptr && roi != nullptr, "PctClip: null argument");
  *out = nullptr;
  HF_CHECK_ARG(min_pct >= 0.f && min_pct <= 100.f && max_pct >= 0.f && max_pct <= 100.f && min_pct < max_pct,
               "PctClip: percentiles must satisfy 0 <= min_pct < max_pct <= 100");
  HF_CHECK_ARG(depth >= 1 && height >= 1 && width >= 1, "PctClip: input must not be empty");
  HF_CHECK_ARG((int64_t)depth * height * width <= INT32_MAX, "PctClip: at most 2^31 - 1 pixels");
  HF_CHECK_ARG(depth <= 65535, "PctClip: at most 65535 slices");
  auto *p = new (std::nothrow) hf_pctclip();
  if (!p)
    return fail(HF_ERR_NOMEM, "PctClip: host allocation failed");
  p->D = depth, p->H = height, p->W = width;
  const size_t n   = (size_t)depth * height * width;
  int         *cnt = nullptr;
  int          rc  = cuda_status(cudaMalloc(&p->mask, n), "PctClip: mask");
  if (rc == HF_OK)
    rc = cuda_status(cudaMalloc(&p->st, sizeof(SelState)), "PctClip: state");
  if (rc == HF_OK)
    rc = cuda_status(cudaMalloc(&cnt, sizeof(int)), "PctClip: count");
  if (rc == HF_OK)
    rc = cuda_status(cudaMemsetAsync(cnt, 0, sizeof(int), s), "PctClip: count");
  if (rc == HF_OK) {
    roi_mask_kernel<<<dim3((width + 15) / 16, (height + 15) / 16, depth), dim3(16, 16), 0, s>>>(
        p->mask, cnt, width, height, depth, roi->cx, roi->cy, roi->rx, roi->ry, roi->angle);
    note_launch();
    rc = launch_status("roi_mask_kernel");
  }
  int count = 0;
  if (rc == HF_OK)
    rc = cuda_status(cudaMemcpyAsync(&count, cnt, sizeof(int), cudaMemcpyDeviceToHost, s), "PctClip: count");
  if (rc == HF_OK)
    rc = cuda_status(cudaStreamSynchronize(s), "PctClip: count");
  cudaFree(cnt);
  if (rc == HF_OK && count <= 0)
    rc = fail(HF_ERR_INVALID, "PctClip: no pixels in ROI");
  if (rc != HF_OK) {
    release(p);
    return rc;
  }
  p->count   = count;
  p->min_idx = (int)(min_pct / 100.0f * (float)(count - 1));
  p->max_idx = (int)(max_pct / 100.0f * (float)(count - 1));
  *out       = p;
  return HF_OK;
}

int hf_pctclip_roi_count(const hf_pctclip *p, int *count) {
  clear_error();
  HF_CHECK_ARG(p != nullptr && count != nullptr, "PctClip: null argument");
  *count = p->count;
  return HF_OK;
}

int hf_pctclip_exec(hf_pctclip *p, const float *in, float *out, float *bounds, hf_stream_t s) {
  clear_error();
  HF_CHECK_ARG(p != nullptr && in != nullptr && out != nullptr, "PctClip: null argument");
  const int64_t n = (int64_t)p->D * p->H * p->W;
  select_init_kernel<<<1, 256, 0, s>>>(p->st, (uint32_t)p->min_idx, (uint32_t)p->max_idx);
  note_launch();
  HF_TRY(launch_status("select_init_kernel"));
  const int grid = grid_for(n, 256 * 8);
  for (int pass = 0; pass < 4; ++pass) {
    select_hist_kernel<<<grid, 256, 0, s>>>(in, p->mask, n, p->st, pass);
    select_step_kernel<<<1, 256, 0, s>>>(p->st, pass);
    note_launch(2);
    HF_TRY(launch_status("select_hist_kernel"));
  }
  clip_kernel<<<grid_for(n), 256, 0, s>>>(in, out, n, p->st);
  note_launch();
  HF_TRY(launch_status("clip_kernel"));
  if (bounds)
    HF_CUDA(cudaMemcpyAsync(bounds, &p->st->lo, 2 * sizeof(float), cudaMemcpyDeviceToDevice, s));
  return HF_OK;
}

int hf_pctclip_destroy(hf_pctclip *p) {
  clear_error();
  release(p);
  return HF_OK;
}

int hf_slideavg_create(int64_t npix, int window, int discard_first, hf_stream_t s, hf_slideavg **out) {
  clear_error();
  HF_CHECK_ARG(out != nullptr, "SlidingAverage: null argument");
  *out = nullptr;
  HF_CHECK_ARG(npix >= 1, "SlidingAverage: image must not be empty");
  HF_CHECK_ARG(window >= 1, "SlidingAverage: window_size must be positive");
  HF_CHECK_ARG(discard_first >= 0, "SlidingAverage: discard_first must be >= 0");
  auto *a = new (std::nothrow) hf_slideavg();
  if (!a)
    return fail(HF_ERR_NOMEM, "SlidingAverage: host allocation failed");
  a->npix = npix, a->window = window, a->discard_first = discard_first;
  int rc = cuda_status(cudaMalloc(&a->ring, (size_t)window * npix * sizeof(float)), "SlidingAverage: ring");
  if (rc == HF_OK)
    rc = cuda_status(cudaMalloc(&a->avg, (size_t)npix * sizeof(float)), "SlidingAverage: average");
  if (rc == HF_OK)
    rc = cuda_status(cudaMemsetAsync(a->ring, 0, (size_t)window * npix * sizeof(float), s), "SlidingAverage: ring");
  if (rc == HF_OK)
    rc = cuda_status(cudaMemsetAsync(a->avg, 0, (size_t)npix * sizeof(float), s), "SlidingAverage: average");
  if (rc != HF_OK) {
    release(a);
    return rc;
  }
  *out = a;
  return HF_OK;
}

int hf_slideavg_push(hf_slideavg *a, const float *in, float *out, int *ready, hf_stream_t s) {
  clear_error();
  HF_CHECK_ARG(a != nullptr && in != nullptr, "SlidingAverage: null argument");
  if (a->discarded < a->discard_first) { // dropped images do not enter the average
    ++a->discarded;
    if (ready)
      *ready = 0;
    return HF_OK;
  }
  slideavg_kernel<<<grid_for(a->npix), 256, 0, s>>>(in, a->ring + (size_t)a->slot * a->npix, a->avg, out, a->npix,
                                                    (float)a->window);
  note_launch();
  HF_TRY(launch_status("slideavg_kernel"));
  a->slot = (a->slot + 1) % a->window;
  ++a->pushes;
  if (ready)
    *ready = a->pushes >= a->window ? 1 : 0;
  return HF_OK;
}

int hf_slideavg_destroy(hf_slideavg *a) {
  clear_error();
  release(a);
  return HF_OK;
}

} // extern "C"
