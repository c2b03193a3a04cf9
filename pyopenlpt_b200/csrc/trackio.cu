// Track files on the device: the rows of STB::saveTracks (src/srcSTB/STB.cpp:967-1004),
// Track::saveTrack (src/srcSTB/Track.cpp:17-26) and Tracer3D::saveObject3D
// (src/srcObject/ObjectInfo.cpp:76-94) formatted by one thread per row -- a length pass,
// an exclusive scan of the lengths, a write pass into one contiguous buffer -- and handed
// to the context's writer thread, which writes the files in posting order while the next
// frame runs.
//
// The numbers are those std::ostream prints with std::fixed and precision 6, i.e. the C
// library's "%.6f": the exact binary value of the double rounded to six decimals, ties
// to even (glibc rounds the exact value in the current rounding mode, round-to-nearest
// here), a leading '-' whenever the sign bit is set ("-0.000000", "-nan").
#include <cmath>
#include <cstdio>
#include <stdexcept>

#include "olpt_ctx.cuh"
#include "olpt_scan.cuh"

namespace olpt {

// ------------------------------------------------------------------ writer thread
void FileWriter::post(std::function<void()> job) {
  std::unique_lock<std::mutex> lk(mu_);
  if (!err_.empty()) {
    std::string e;
    e.swap(err_);
    throw ApiError{OLPT_ERR_INVALID_ARG, e};
  }
  if (!th_.joinable()) {
    quit_ = false;
    th_ = std::thread([this] { loop(); });
  }
  q_.push_back(std::move(job));
  cv_.notify_one();
}

std::string FileWriter::wait() {
  std::unique_lock<std::mutex> lk(mu_);
  idle_cv_.wait(lk, [this] { return q_.empty() && !busy_; });
  std::string e;
  e.swap(err_);
  return e;
}

void FileWriter::stop() {
  {
    std::unique_lock<std::mutex> lk(mu_);
    if (!th_.joinable()) return;
    quit_ = true;
    cv_.notify_one();
  }
  th_.join();
}

void FileWriter::loop() {
  std::unique_lock<std::mutex> lk(mu_);
  for (;;) {
    cv_.wait(lk, [this] { return quit_ || !q_.empty(); });
    if (q_.empty()) return;  // quit with nothing left to write
    std::function<void()> job = std::move(q_.front());
    q_.pop_front();
    busy_ = true;
    lk.unlock();
    std::string e;
    try {
      job();
    } catch (const std::exception& x) {
      e = x.what();
    } catch (const ApiError& x) {
      e = x.msg;
    } catch (...) {
      e = "track file writer: unknown error";
    }
    lk.lock();
    if (!e.empty() && err_.empty()) err_ = e;
    busy_ = false;
    if (q_.empty()) idle_cv_.notify_all();
  }
}

namespace {

// ------------------------------------------------------------------ number formatting
struct Fixed6 {
  unsigned long long ip;  // integer part after rounding
  int frac;               // the six decimals
  int neg;                // sign bit
  int kind;               // 0 finite, 1 NaN, 2 infinite, 3 |v| >= 2^63 (not formatted)
};

__device__ Fixed6 fixed6(double v) {
  Fixed6 r{0ull, 0, (int)((unsigned long long)__double_as_longlong(v) >> 63), 0};
  if (isnan(v)) {
    r.kind = 1;
    return r;
  }
  if (isinf(v)) {
    r.kind = 2;
    return r;
  }
  const double a = fabs(v);
  if (!(a < 9223372036854775808.0)) {
    r.kind = 3;
    return r;
  }
  const double ip = floor(a);
  const double f = a - ip;                // exact (both on a's grid)
  const double p = f * 1e6;               // rounded product, < 2^20: ulp(p) <= 2^-33
  const double e = __fma_rn(f, 1e6, -p);  // its exact error: f * 10^6 = p + e
  const double q = floor(p);
  const double d = p - q;                 // exact; a multiple of ulp(p), so is 0.5
  // d != 0.5: |e| <= ulp(p) / 2 cannot carry p + e across q + 1/2; d == 0.5: e decides,
  // a true tie (e == 0) goes to the even neighbour
  const bool up = d > 0.5 || (d == 0.5 && (e > 0.0 || (e == 0.0 && fmod(q, 2.0) != 0.0)));
  long long fr = (long long)q + (up ? 1 : 0);
  unsigned long long I = (unsigned long long)ip;
  if (fr >= 1000000) {
    fr -= 1000000;
    ++I;
  }
  r.ip = I;
  r.frac = (int)fr;
  return r;
}

__device__ __forceinline__ int u64_len(unsigned long long x) {
  int n = 1;
  while (x >= 10ull) {
    x /= 10ull;
    ++n;
  }
  return n;
}

__device__ __forceinline__ char* put_u64(char* o, unsigned long long x) {
  const int n = u64_len(x);
  for (int i = n - 1; i >= 0; --i) {
    o[i] = (char)('0' + (int)(x % 10ull));
    x /= 10ull;
  }
  return o + n;
}

__device__ __forceinline__ int int_len(int v) {
  return v < 0 ? 1 + u64_len(0ull - (unsigned long long)(long long)v)
               : u64_len((unsigned long long)v);
}

__device__ __forceinline__ char* put_int(char* o, int v) {
  if (v < 0) {
    *o++ = '-';
    return put_u64(o, 0ull - (unsigned long long)(long long)v);
  }
  return put_u64(o, (unsigned long long)v);
}

__device__ __forceinline__ int fixed6_len(const Fixed6& f) {
  if (f.kind == 1 || f.kind == 2) return f.neg + 3;
  return f.neg + u64_len(f.ip) + 7;
}

__device__ __forceinline__ char* put_fixed6(char* o, const Fixed6& f) {
  if (f.neg) *o++ = '-';
  if (f.kind == 1 || f.kind == 2) {
    const char* w = f.kind == 1 ? "nan" : "inf";
    o[0] = w[0];
    o[1] = w[1];
    o[2] = w[2];
    return o + 3;
  }
  o = put_u64(o, f.ip);
  *o++ = '.';
  int x = f.frac;
  for (int i = 5; i >= 0; --i) {
    o[i] = (char)('0' + x % 10);
    x /= 10;
  }
  return o + 6;
}

// ------------------------------------------------------------------ rows
// Row i: ints[i * n_int + k] (k < n_int), then d1[i * n1 + k] (k < n1), then
// d2[i * n2 + k] (k < n2), comma separated, ended by '\n'.
struct Rows {
  const int* ints;
  const double* d1;
  const double* d2;
  int n_int, n1, n2;
  int64_t n;
  __device__ double dbl(int64_t i, int k) const {
    return k < n1 ? d1[i * n1 + k] : d2[i * n2 + (k - n1)];
  }
};

__global__ void row_len_kernel(const Rows r, int* len, int* bad) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= r.n) return;
  int L = 0, fields = 0;
  for (int k = 0; k < r.n_int; ++k, ++fields) L += int_len(r.ints[i * r.n_int + k]);
  bool out_of_range = false;
  for (int k = 0; k < r.n1 + r.n2; ++k, ++fields) {
    const Fixed6 f = fixed6(r.dbl(i, k));
    out_of_range |= f.kind == 3;
    L += fixed6_len(f);
  }
  L += fields > 0 ? fields - 1 : 0;  // separators
  len[i] = L + 1;                     // newline
  if (out_of_range) atomicAdd(bad, 1);
}

__global__ void row_put_kernel(const Rows r, const int* off, char* out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= r.n) return;
  char* o = out + off[i];
  bool first = true;
  for (int k = 0; k < r.n_int; ++k) {
    if (!first) *o++ = ',';
    first = false;
    o = put_int(o, r.ints[i * r.n_int + k]);
  }
  for (int k = 0; k < r.n1 + r.n2; ++k) {
    if (!first) *o++ = ',';
    first = false;
    o = put_fixed6(o, fixed6(r.dbl(i, k)));
  }
  *o = '\n';
}

inline int blocks(int64_t n) { return (int)((n + 255) / 256); }

}  // namespace

// Rows [0, n) (device arrays as in Rows) formatted on the device and appended to out.
// n is at most kMaxRowsPerPass, so every offset fits an int.
void format_rows_device(olpt_ctx* ctx, const int* ints, int n_int, const double* d1, int n1,
                        const double* d2, int n2, int64_t n, std::string& out) {
  if (n <= 0) return;
  OLPT_REQUIRE(n <= kMaxRowsPerPass, OLPT_ERR_INVALID_ARG, "too many rows in one pass");
  OLPT_REQUIRE(n_int + n1 + n2 <= 64, OLPT_ERR_INVALID_ARG, "too many fields per row");
  cudaStream_t s = ctx->stream;
  TrackIoWork& W = ctx->tio;
  W.len.ensure((size_t)(n + 1) * sizeof(int), s);
  W.off.ensure((size_t)(n + 1) * sizeof(int), s);
  W.bad.ensure(sizeof(int) * 2, s);
  OLPT_CUDA(cudaMemsetAsync(W.bad.p, 0, sizeof(int), s));
  const Rows r{ints, d1, d2, n_int, n1, n2, n};
  row_len_kernel<<<OLPT_G(blocks(n)), 256, 0, s>>>(r, W.len.as<int>(), W.bad.as<int>());
  OLPT_CUDA(cudaGetLastError());
  exclusive_scan(W.len.as<int>(), (int)n, W.off.as<int>(), W.tmp, s);
  int hdr[2] = {0, 0};
  OLPT_CUDA(cudaMemcpyAsync(&hdr[0], W.off.as<int>() + n, sizeof(int), cudaMemcpyDeviceToHost, s));
  OLPT_CUDA(cudaMemcpyAsync(&hdr[1], W.bad.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  OLPT_CUDA(cudaStreamSynchronize(s));
  OLPT_REQUIRE(hdr[1] == 0, OLPT_ERR_UNSUPPORTED,
               "a value of magnitude 2^63 or more cannot be written to a track file");
  const size_t total = (size_t)hdr[0];
  W.bytes.ensure(total + 16, s);
  row_put_kernel<<<OLPT_G(blocks(n)), 256, 0, s>>>(r, W.off.as<int>(), W.bytes.as<char>());
  OLPT_CUDA(cudaGetLastError());
  const size_t at = out.size();
  out.resize(at + total);
  OLPT_CUDA(cudaMemcpyAsync(&out[at], W.bytes.p, total, cudaMemcpyDeviceToHost, s));
  OLPT_CUDA(cudaStreamSynchronize(s));
}

// Writes `bytes` to `file` on the writer thread (now, when async is off).
void write_file(olpt_ctx* ctx, const std::string& file, std::string&& bytes) {
  auto job = [file, b = std::move(bytes)]() {
    std::FILE* f = std::fopen(file.c_str(), "w");
    if (!f) throw std::runtime_error("Cannot open file: " + file);
    const size_t put = b.empty() ? 0 : std::fwrite(b.data(), 1, b.size(), f);
    const bool ok = (put == b.size()) & (std::fclose(f) == 0);
    if (!ok) throw std::runtime_error("Cannot write file: " + file);
  };
  ctx->tio.writer.post(std::move(job));
  if (!ctx->tio.async) flush_files(ctx);
}

void flush_files(olpt_ctx* ctx) {
  const std::string e = ctx->tio.writer.wait();
  OLPT_REQUIRE(e.empty(), OLPT_ERR_INVALID_ARG, e);
}

}  // namespace olpt
