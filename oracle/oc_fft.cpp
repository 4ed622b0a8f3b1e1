// Double-precision FFT for the CPU oracle.  See oc_fft.hpp for conventions.
#include "oc_fft.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>

namespace oc {

namespace {

const double kPi = 3.14159265358979323846264338327950288;

int smallest_factor(int n) {
  for (int r : {4, 2, 3, 5, 7}) {
    if (n % r == 0) return r;
  }
  return n;  // prime (or has only large prime factors)
}

bool is_smooth(int n) {
  while (n % 2 == 0) n /= 2;
  while (n % 3 == 0) n /= 3;
  while (n % 5 == 0) n /= 5;
  while (n % 7 == 0) n /= 7;
  return n == 1;
}

void bluestein(cd* x, int n, int sign);

// Recursive mixed-radix decimation in time over smooth sizes.
void mixed_radix(cd* x, int n, int sign, std::vector<cd>& scratch) {
  if (n == 1) return;
  int r = smallest_factor(n);
  if (r == n && n > 7) {
    bluestein(x, n, sign);
    return;
  }
  int m = n / r;
  // gather the r decimated subsequences
  std::vector<cd> sub(n);
  for (int q = 0; q < r; ++q)
    for (int j = 0; j < m; ++j) sub[q * m + j] = x[j * r + q];
  for (int q = 0; q < r; ++q) mixed_radix(&sub[q * m], m, sign, scratch);
  // butterflies: X[k + m s] = sum_q sub_q[k] w_n^{q (k + m s)}
  const double ang = sign * 2.0 * kPi / n;
  for (int k = 0; k < m; ++k) {
    for (int s = 0; s < r; ++s) {
      int kk = k + m * s;
      cd acc(0.0, 0.0);
      for (int q = 0; q < r; ++q) {
        long long e = (long long)q * kk % n;
        double a = ang * (double)e;
        acc += sub[q * m + k] * cd(std::cos(a), std::sin(a));
      }
      x[kk] = acc;
    }
  }
}

int next_pow2(int n) {
  int p = 1;
  while (p < n) p <<= 1;
  return p;
}

void bluestein(cd* x, int n, int sign) {
  int m = next_pow2(2 * n - 1);
  std::vector<cd> w(n), a(m, cd(0, 0)), b(m, cd(0, 0));
  for (int k = 0; k < n; ++k) {
    long long k2 = (long long)k * k % (2LL * n);
    double ang = sign * kPi * (double)k2 / n;
    w[k] = cd(std::cos(ang), std::sin(ang));
  }
  for (int k = 0; k < n; ++k) a[k] = x[k] * w[k];
  b[0] = std::conj(w[0]);
  for (int k = 1; k < n; ++k) {
    b[k] = std::conj(w[k]);
    b[m - k] = std::conj(w[k]);
  }
  fft_c2c(a.data(), m, -1);
  fft_c2c(b.data(), m, -1);
  for (int k = 0; k < m; ++k) a[k] *= b[k];
  fft_c2c(a.data(), m, +1);
  for (int k = 0; k < n; ++k) x[k] = a[k] / (double)m * w[k];
}

// Iterative radix-2 with a cached twiddle table for powers of two.
struct Pow2Plan {
  int n;
  std::vector<cd> tw;  // exp(-2 pi i k / n), k < n/2
  std::vector<int> rev;
};

std::mutex g_plan_mutex;
std::map<int, std::shared_ptr<Pow2Plan>> g_plans;

std::shared_ptr<Pow2Plan> get_plan(int n) {
  std::lock_guard<std::mutex> lock(g_plan_mutex);
  auto it = g_plans.find(n);
  if (it != g_plans.end()) return it->second;
  auto p = std::make_shared<Pow2Plan>();
  p->n = n;
  p->tw.resize(n / 2 > 0 ? n / 2 : 1);
  for (int k = 0; k < n / 2; ++k) {
    double a = -2.0 * kPi * k / n;
    p->tw[k] = cd(std::cos(a), std::sin(a));
  }
  p->rev.resize(n);
  int lg = 0;
  while ((1 << lg) < n) ++lg;
  for (int i = 0; i < n; ++i) {
    int r = 0;
    for (int b = 0; b < lg; ++b)
      if (i & (1 << b)) r |= 1 << (lg - 1 - b);
    p->rev[i] = r;
  }
  g_plans[n] = p;
  return p;
}

void radix2(cd* x, int n, int sign) {
  auto p = get_plan(n);
  for (int i = 0; i < n; ++i)
    if (i < p->rev[i]) std::swap(x[i], x[p->rev[i]]);
  for (int len = 2; len <= n; len <<= 1) {
    int half = len / 2;
    int step = n / len;
    for (int i = 0; i < n; i += len) {
      for (int j = 0; j < half; ++j) {
        cd w = p->tw[j * step];
        if (sign > 0) w = std::conj(w);
        cd u = x[i + j];
        cd v = x[i + j + half] * w;
        x[i + j] = u + v;
        x[i + j + half] = u - v;
      }
    }
  }
}

}  // namespace

void fft_c2c(cd* data, int n, int sign) {
  if (n <= 1) return;
  if ((n & (n - 1)) == 0) {
    radix2(data, n, sign);
    return;
  }
  if (!is_smooth(n) && smallest_factor(n) == n) {
    bluestein(data, n, sign);
    return;
  }
  std::vector<cd> scratch;
  mixed_radix(data, n, sign, scratch);
}

// Perturbation of every transform's output at the size of single-precision
// rounding (a sensitivity probe, off unless a test sets a seed): each output value
// v becomes v (1 + e), |e| <= 2^-24 sqrt(log2 n), e drawn from a hash of the seed,
// the value's bits and its index, so it is deterministic and thread-safe.
static unsigned long long g_perturb_seed = 0;

static double perturb_factor(double v, size_t k, int n) {
  unsigned long long h;
  std::memcpy(&h, &v, sizeof(h));
  h ^= g_perturb_seed * 0x9E3779B97F4A7C15ull + (unsigned long long)k * 0xBF58476D1CE4E5B9ull;
  h ^= h >> 31;
  h *= 0x94D049BB133111EBull;
  h ^= h >> 29;
  const double u = (double)(h >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
  return 1.0 + u * std::ldexp(1.0, -24) * std::sqrt(std::log2((double)std::max(n, 2)));
}

static void perturb(cd* x, size_t m, int n) {
  if (!g_perturb_seed) return;
  for (size_t k = 0; k < m; ++k)
    x[k] = cd(x[k].real() * perturb_factor(x[k].real(), 2 * k, n),
              x[k].imag() * perturb_factor(x[k].imag(), 2 * k + 1, n));
}

static void perturb(double* x, size_t m, int n) {
  if (!g_perturb_seed) return;
  for (size_t k = 0; k < m; ++k) x[k] *= perturb_factor(x[k], k, n);
}

void fft_r2c_1d(const double* in, cd* out, int n) {
  std::vector<cd> buf(n);
  for (int i = 0; i < n; ++i) buf[i] = cd(in[i], 0.0);
  fft_c2c(buf.data(), n, -1);
  for (int k = 0; k <= n / 2; ++k) out[k] = buf[k];
  perturb(out, n / 2 + 1, n);
}

void fft_c2r_1d(const cd* in, double* out, int n) {
  std::vector<cd> buf(n);
  int h = n / 2;
  for (int k = 0; k <= h; ++k) buf[k] = in[k];
  for (int k = h + 1; k < n; ++k) buf[k] = std::conj(in[n - k]);
  // Hermitian completion treats the self-conjugate bins as real, like a C2R.
  buf[0] = cd(in[0].real(), 0.0);
  if (n % 2 == 0) buf[h] = cd(in[h].real(), 0.0);
  fft_c2c(buf.data(), n, +1);
  for (int i = 0; i < n; ++i) out[i] = buf[i].real();
  perturb(out, n, n);
}

void fft_r2c_2d(const double* in, int in_stride, cd* out, int nx, int ny) {
  int cx = nx / 2 + 1;
  for (int y = 0; y < ny; ++y) fft_r2c_1d(in + (size_t)y * in_stride, out + (size_t)y * cx, nx);
  std::vector<cd> col(ny);
  for (int x = 0; x < cx; ++x) {
    for (int y = 0; y < ny; ++y) col[y] = out[(size_t)y * cx + x];
    fft_c2c(col.data(), ny, -1);
    for (int y = 0; y < ny; ++y) out[(size_t)y * cx + x] = col[y];
  }
}

void fft_c2r_2d(const cd* in, double* out, int out_stride, int nx, int ny) {
  int cx = nx / 2 + 1;
  std::vector<cd> tmp((size_t)cx * ny);
  std::vector<cd> col(ny);
  for (int x = 0; x < cx; ++x) {
    for (int y = 0; y < ny; ++y) col[y] = in[(size_t)y * cx + x];
    fft_c2c(col.data(), ny, +1);
    for (int y = 0; y < ny; ++y) tmp[(size_t)y * cx + x] = col[y];
  }
  for (int y = 0; y < ny; ++y) fft_c2r_1d(&tmp[(size_t)y * cx], out + (size_t)y * out_stride, nx);
}

}  // namespace oc

extern "C" void oc_fft_perturb(unsigned long long seed) { oc::g_perturb_seed = seed; }

// Checked against numpy in the oracle's own tests.
extern "C" void oc_rfft(const double* in, double* out_re_im, int n) {
  std::vector<oc::cd> spec(n / 2 + 1);
  oc::fft_r2c_1d(in, spec.data(), n);
  for (int k = 0; k <= n / 2; ++k) {
    out_re_im[2 * k] = spec[k].real();
    out_re_im[2 * k + 1] = spec[k].imag();
  }
}

extern "C" void oc_rfft2(const double* in, double* out_re_im, int nx, int ny) {
  std::vector<oc::cd> spec((size_t)(nx / 2 + 1) * ny);
  oc::fft_r2c_2d(in, nx, spec.data(), nx, ny);
  for (size_t k = 0; k < spec.size(); ++k) {
    out_re_im[2 * k] = spec[k].real();
    out_re_im[2 * k + 1] = spec[k].imag();
  }
}

extern "C" void oc_irfft2(const double* in_re_im, double* out, int nx, int ny) {
  std::vector<oc::cd> spec((size_t)(nx / 2 + 1) * ny);
  for (size_t k = 0; k < spec.size(); ++k) spec[k] = oc::cd(in_re_im[2 * k], in_re_im[2 * k + 1]);
  oc::fft_c2r_2d(spec.data(), out, nx, nx, ny);
}
