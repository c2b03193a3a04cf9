// OTF::estimateUniformOTFFromImage (src/srcSTB/OTF.cpp:17-144) on the device: the
// tracer detections of the context's planes (the images of one camera), at most 1000 of
// them per image chosen by the reference's seeded std::shuffle, the window samples
// around each detection gathered on the device, and the least squares
//   a = min(mean(I_c) + 2 std(I_c), max(I_c)),
//   (b, c) = inverse(C^T C) C^T L,  C_k = ((col - xc)^2, (row - yc)^2),
//   L_k = -log(max(I_k, 1e-4)) + log(a)
// reduced on the device in the reference's summation order (each sum is one dependent
// chain, so the result is the reference's to the last bit).
//
// What the C library computes in the reference is computed by it here too, because
// CUDA's pow and log round differently in the last bit (the C library's pow(x, 2) is not
// always x * x either): the squares std::pow(col - xc, 2) (one per window column and
// row of a detection), the statistics of a over the at most 1000 a-samples per image
// (their std::pow(d, 2)), log(a), and log(I) of samples that are not integer levels
// (integer levels use the library's log table of the detection kernel).  The random
// permutation is the reference's minstd_rand0 sequence run on the host; it depends only
// on the detection count.
#include <algorithm>
#include <cmath>
#include <random>

#include "olpt_ctx.cuh"
#include "olpt_scan.cuh"

namespace olpt {

void find_peaks_device(olpt_ctx* ctx, double min_int, bool sync_counts);
void ensure_log_luts(olpt_ctx* ctx);

namespace {

struct PlaneRef {
  const unsigned char* p;
  int dtype;
  int64_t pitch;
};

struct PlaneSet {
  PlaneRef pl[OLPT_MAX_CAM];
};

__device__ __forceinline__ double plane_at(const PlaneRef& P, int r, int c) {
  const unsigned char* row = P.p + (int64_t)r * P.pitch;
  switch (P.dtype) {
    case OLPT_U8: return (double)row[c];
    case OLPT_U16: return (double)reinterpret_cast<const uint16_t*>(row)[c];
    case OLPT_F32: return (double)reinterpret_cast<const float*>(row)[c];
    default: return reinterpret_cast<const double*>(row)[c];
  }
}

// One detection's window (row-major samples) and the reference's a-sample.
struct Win {
  int plane, rmin, rmax, cmin, cmax, yc0, xc0;
  int64_t off;     // first sample
  int64_t pw_off;  // first column square; the row squares follow the column ones
};

// one warp per detection: the a-sample, then the window's samples in row-major order
__global__ void gather_kernel(const PlaneSet ps, const Win* win, int n_win, const double* pw,
                              double* a_list, double* I, double* cx, double* cy) {
  const int w = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (w >= n_win) return;
  const Win W = win[w];
  const PlaneRef& P = ps.pl[W.plane];
  if (lane == 0) a_list[w] = plane_at(P, W.yc0, W.xc0);
  const int nc = W.cmax - W.cmin, nr = W.rmax - W.rmin;
  for (int k = lane; k < nr * nc; k += 32) {
    const int r = k / nc, c = k % nc;
    I[W.off + k] = plane_at(P, W.rmin + r, W.cmin + c);
    cx[W.off + k] = pw[W.pw_off + c];
    cy[W.off + k] = pw[W.pw_off + nc + r];
  }
}

// log(max(I, 1e-4)) through the log table where I is an integer level of it; other
// samples are marked (the host fills them with the C library's log)
__global__ void log_kernel(const double* I, int64_t n, const double* lut, int lut_n, double* logI,
                           int* n_other) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= n) return;
  const double v = I[k];
  const bool level = v >= 0.0 && v <= (double)(lut_n - 1) && v == floor(v);
  if (level) {
    logI[k] = lut[(int)v];
  } else if (v < 1e-4) {
    logI[k] = lut[0];  // log(1e-4), the reference's floor
  } else {
    logI[k] = __longlong_as_double(0x7ff8000000000001LL);  // filled on the host
    atomicAdd(n_other, 1);
  }
}

// C^T C summed in sample order (Matrix::operator*: from 0, index order), one thread
// per dependent chain: A00, A01 (= A10: the products commute), A11.
__global__ void normal_kernel(const double* cx, const double* cy, int64_t n, double* out) {
  const int t = threadIdx.x;
  if (t > 2) return;
  const double* u = (t == 2) ? cy : cx;
  const double* v = (t == 0) ? cx : cy;
  double s = 0.0;
  for (int64_t i = 0; i < n; ++i) s += u[i] * v[i];
  out[t] = s;
}

// coef_r = sum_k (0 + inv[r][0] cx_k + inv[r][1] cy_k) * (-logI_k + log_a), k in order
__global__ void coef_kernel(const double* cx, const double* cy, const double* logI, int64_t n,
                            double inv00, double inv01, double inv10, double inv11, double log_a,
                            double* out) {
  const int r = threadIdx.x;
  if (r > 1) return;
  const double i0 = r ? inv10 : inv00, i1 = r ? inv11 : inv01;
  double s = 0.0;
  for (int64_t k = 0; k < n; ++k) {
    double q = 0.0;
    q += i0 * cx[k];
    q += i1 * cy[k];
    s += q * (-logI[k] + log_a);
  }
  out[r] = s;
}

int blocks(int64_t n, int t = 256) { return (int)((n + t - 1) / t); }

}  // namespace

// myMATH::inverse of a 2 x 2 (src/srcMath/myMATH.cpp, Gauss-Jordan with scaled partial
// pivoting) in the reference's operation order.
void gauss_inverse2(const double A[4], double inv[4]) {
  double u[4] = {A[0], A[1], A[2], A[3]};
  int idx[2] = {0, 1};
  const double maxrow[2] = {std::max(u[0], u[1]), std::max(u[2], u[3])};
  double mp = 0;
  int t = 0;
  for (int x = 0; x < 2; ++x) {
    const double piv = std::fabs(u[2 * idx[x]] / maxrow[idx[x]]);
    if (piv > mp) {
      mp = piv;
      t = x;
    }
  }
  std::swap(idx[t], idx[0]);
  const double m = u[2 * idx[1]] / u[2 * idx[0]];
  u[2 * idx[1]] = m;
  u[2 * idx[1] + 1] -= m * u[2 * idx[0] + 1];
  double bm[4] = {1, 0, 0, 1};
  for (int it = 0; it < 2; ++it) {
    bm[2 * idx[1] + it] -= u[2 * idx[1]] * bm[2 * idx[0] + it];
    inv[2 + it] = bm[2 * idx[1] + it] / u[2 * idx[1] + 1];
    double z = bm[2 * idx[0] + it];
    z -= u[2 * idx[0] + 1] * inv[2 + it];
    inv[it] = z / u[2 * idx[0]];
  }
}

// a, b, c of the context's planes; false when an image has no detection (the reference
// then leaves the OTF as it is).
bool otf_estimate_device(olpt_ctx* ctx, double min_int, double r_pt, int max_det, double abc[3],
                         int64_t* n_samples) {
  cudaStream_t s = ctx->stream;
  const int n_img = ctx->n_cam;
  OLPT_REQUIRE(n_img >= 1, OLPT_ERR_INVALID_ARG, "no images uploaded");
  find_peaks_device(ctx, min_int, true);
  ensure_log_luts(ctx);
  // the chosen detections per image: std::shuffle(list, default_random_engine(123)),
  // then the first max_det (OTF.cpp:41-46); the permutation depends only on the count
  std::vector<std::vector<int>> chosen(n_img);
  for (int p = 0; p < n_img; ++p) {
    const int64_t cnt = ctx->det_counts_h[p];
    if (cnt == 0) {
      *n_samples = 0;
      return false;
    }
    std::vector<int> idx((size_t)cnt);
    for (int64_t i = 0; i < cnt; ++i) idx[i] = (int)i;
    if (cnt > max_det) {
      std::shuffle(idx.begin(), idx.end(), std::default_random_engine(123));
      idx.resize((size_t)max_det);
    }
    chosen[p] = std::move(idx);
  }
  // the chosen centres, their windows and the C library's squares of the offsets
  std::vector<Win> wins;
  std::vector<double> pw;
  int64_t n = 0;
  for (int p = 0; p < n_img; ++p) {
    const int64_t cnt = ctx->det_counts_h[p];
    std::vector<double> hx(cnt), hy(cnt);
    OLPT_CUDA(cudaMemcpyAsync(hx.data(), ctx->dets[p].x.p, cnt * 8, cudaMemcpyDeviceToHost, s));
    OLPT_CUDA(cudaMemcpyAsync(hy.data(), ctx->dets[p].y.p, cnt * 8, cudaMemcpyDeviceToHost, s));
    OLPT_CUDA(cudaStreamSynchronize(s));
    const int n_row = ctx->img[p].H, n_col = ctx->img[p].W;
    for (int j : chosen[p]) {
      const double xc = hx[j], yc = hy[j];
      Win w;
      w.plane = p;
      w.yc0 = std::clamp<int>(int(std::round(yc)), 0, n_row - 1);
      w.xc0 = std::clamp<int>(int(std::round(xc)), 0, n_col - 1);
      w.rmin = std::max(0, int(std::floor(yc - r_pt)));
      w.rmax = std::min(n_row, int(std::ceil(yc + r_pt + 1)));
      w.cmin = std::max(0, int(std::floor(xc - r_pt)));
      w.cmax = std::min(n_col, int(std::ceil(xc + r_pt + 1)));
      w.off = n;
      w.pw_off = (int64_t)pw.size();
      for (int col = w.cmin; col < w.cmax; ++col) pw.push_back(std::pow(col - xc, 2));
      for (int row = w.rmin; row < w.rmax; ++row) pw.push_back(std::pow(row - yc, 2));
      n += (int64_t)std::max(0, w.rmax - w.rmin) * std::max(0, w.cmax - w.cmin);
      wins.push_back(w);
    }
  }
  const int n_win = (int)wins.size();
  PlaneSet ps{};
  for (int p = 0; p < n_img; ++p)
    ps.pl[p] = PlaneRef{ctx->img[p].buf.as<unsigned char>(), ctx->img[p].dtype, ctx->img[p].pitch};
  DevBuf& B = ctx->scratch;
  // layout: wins | pw | a-samples | I | cx | cy | logI | sums (8) | count of other logs
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  const size_t o_win = 0, o_pw = al(o_win + wins.size() * sizeof(Win));
  const size_t o_a = al(o_pw + pw.size() * 8), o_I = al(o_a + (size_t)n_win * 8);
  const size_t o_cx = al(o_I + (size_t)n * 8), o_cy = al(o_cx + (size_t)n * 8);
  const size_t o_log = al(o_cy + (size_t)n * 8), o_out = al(o_log + (size_t)n * 8);
  const size_t o_cnt = al(o_out + 8 * 8), total = o_cnt + 16;
  B.ensure(total, s);
  unsigned char* b = B.as<unsigned char>();
  Win* d_win = reinterpret_cast<Win*>(b + o_win);
  double* d_pw = reinterpret_cast<double*>(b + o_pw);
  double* d_a = reinterpret_cast<double*>(b + o_a);
  double* d_I = reinterpret_cast<double*>(b + o_I);
  double* d_cx = reinterpret_cast<double*>(b + o_cx);
  double* d_cy = reinterpret_cast<double*>(b + o_cy);
  double* d_log = reinterpret_cast<double*>(b + o_log);
  double* d_out = reinterpret_cast<double*>(b + o_out);
  int* d_cnt = reinterpret_cast<int*>(b + o_cnt);
  OLPT_CUDA(cudaMemcpyAsync(d_win, wins.data(), wins.size() * sizeof(Win), cudaMemcpyHostToDevice, s));
  if (!pw.empty())
    OLPT_CUDA(cudaMemcpyAsync(d_pw, pw.data(), pw.size() * 8, cudaMemcpyHostToDevice, s));
  OLPT_CUDA(cudaMemsetAsync(d_cnt, 0, sizeof(int), s));
  gather_kernel<<<OLPT_G(blocks((int64_t)n_win * 32)), 256, 0, s>>>(ps, d_win, n_win, d_pw, d_a,
                                                                    d_I, d_cx, d_cy);
  OLPT_CUDA(cudaGetLastError());
  // integer-level planes use the 16-bit table, float planes too for their integer samples
  if (n > 0)
    log_kernel<<<OLPT_G(blocks(n)), 256, 0, s>>>(d_I, n, ctx->lut_u16.as<double>(), 65536, d_log,
                                                 d_cnt);
  normal_kernel<<<OLPT_G(1), 32, 0, s>>>(d_cx, d_cy, n, d_out);
  OLPT_CUDA(cudaGetLastError());
  double nm[3];
  int n_other = 0;
  std::vector<double> a_list(n_win);
  OLPT_CUDA(cudaMemcpyAsync(nm, d_out, sizeof nm, cudaMemcpyDeviceToHost, s));
  OLPT_CUDA(cudaMemcpyAsync(&n_other, d_cnt, sizeof(int), cudaMemcpyDeviceToHost, s));
  OLPT_CUDA(cudaMemcpyAsync(a_list.data(), d_a, n_win * 8, cudaMemcpyDeviceToHost, s));
  OLPT_CUDA(cudaStreamSynchronize(s));
  if (n_other > 0) {  // samples that are not integer levels: the C library's log
    std::vector<double> hI(n), hl(n);
    OLPT_CUDA(cudaMemcpyAsync(hI.data(), d_I, n * 8, cudaMemcpyDeviceToHost, s));
    OLPT_CUDA(cudaMemcpyAsync(hl.data(), d_log, n * 8, cudaMemcpyDeviceToHost, s));
    OLPT_CUDA(cudaStreamSynchronize(s));
    for (int64_t k = 0; k < n; ++k)
      if (std::isnan(hl[k])) hl[k] = std::log(hI[k]);
    OLPT_CUDA(cudaMemcpyAsync(d_log, hl.data(), n * 8, cudaMemcpyHostToDevice, s));
  }
  // a = min(mean + 2 std, max) over the a-samples (OTF.cpp:99-111)
  const double a_max = *std::max_element(a_list.begin(), a_list.end());
  double a_mean = 0, a_std = 0;
  for (int i = 0; i < n_win; ++i) a_mean += a_list[i];
  a_mean /= n_win;
  for (int i = 0; i < n_win; ++i) a_std += std::pow(a_list[i] - a_mean, 2);
  a_std = std::sqrt(a_std / n_win);
  const double a = std::min(a_mean + 2 * a_std, a_max);
  double A[4] = {nm[0], nm[1], nm[1], nm[2]}, inv[4];
  gauss_inverse2(A, inv);
  coef_kernel<<<OLPT_G(1), 32, 0, s>>>(d_cx, d_cy, d_log, n, inv[0], inv[1], inv[2], inv[3],
                                       std::log(a), d_out + 4);
  OLPT_CUDA(cudaGetLastError());
  double coef[2];
  OLPT_CUDA(cudaMemcpyAsync(coef, d_out + 4, sizeof coef, cudaMemcpyDeviceToHost, s));
  OLPT_CUDA(cudaStreamSynchronize(s));
  abc[0] = a;
  abc[1] = coef[0];
  abc[2] = coef[1];
  *n_samples = n;
  return true;
}

}  // namespace olpt
