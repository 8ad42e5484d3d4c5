// C ABI (include/mpir_b200.h).  Every entry point converts exceptions into
// status codes and keeps the message for mpir_last_error().
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/mpir_b200.h"
#include "group.hpp"
#include "server.hpp"
#include "solver.hpp"

namespace mpir {

struct StatusError : std::runtime_error {
  int code;
  StatusError(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

static thread_local std::string g_err;

template <class F>
static auto guard(F &&f) -> decltype(f()) {
  try {
    g_err.clear();
    return f();
  } catch (const StatusError &e) {
    g_err = e.what();
    return e.code;
  } catch (const WaitTimeout &e) {
    g_err = e.what();
    return MPIR_ERR_TIMEOUT;
  } catch (const CudaError &e) {
    g_err = e.what();
    return e.code == cudaErrorMemoryAllocation ? MPIR_ERR_NOMEM : MPIR_ERR_CUDA;
  } catch (const std::bad_alloc &) {
    g_err = "host allocation failed";
    return MPIR_ERR_NOMEM;
  } catch (const std::invalid_argument &e) {
    g_err = e.what();
    return MPIR_ERR_ARGUMENT;
  } catch (const std::logic_error &e) {
    g_err = e.what();
    return MPIR_ERR_STATE;
  } catch (const std::exception &e) {
    g_err = e.what();
    return MPIR_ERR_CUDA;
  }
}

// Row-by-row etree reach (the symbolic half of qdldl.hpp:228-326): row k of
// L holds the tree paths from each i with A(i,k) != 0 up to k.  Appending k
// to each visited column gives QDLDL's Li order (rows ascending).
static void exact_pattern(const Symbolic &S, std::vector<int64_t> &Lp,
                          std::vector<int64_t> &Li) {
  const int64_t n = S.n;
  Lp.assign(n + 1, 0);
  for (int64_t j = 0; j < n; j++) Lp[j + 1] = Lp[j] + S.Lnz[j];
  Li.resize(Lp[n]);
  std::vector<int64_t> next(Lp.begin(), Lp.end() - 1), mark(n, -1);
  for (int64_t k = 0; k < n; k++) {
    mark[k] = k;
    for (int64_t p = S.Cp[k]; p < S.Cp[k + 1]; p++)
      for (int64_t i = S.Ci[p]; mark[i] != k; i = S.etree[i]) {
        Li[next[i]++] = k;
        mark[i]       = k;
      }
  }
}

// Local row of global row r in supernode J's index set.
static int64_t local_row(const Symbolic &S, int64_t J, int64_t r) {
  const int64_t f = S.sfirst[J], l = S.sfirst[J + 1], w = l - f;
  if (r < l) return r - f;
  const int32_t *b = S.srows.data() + S.srowptr[J] + w;
  const int32_t *e = S.srows.data() + S.srowptr[J + 1];
  const int32_t *it = std::lower_bound(b, e, static_cast<int32_t>(r));
  if (it == e || *it != r) return -1;
  return w + (it - b);
}

// Copy the factor out of the panels into QDLDL's CSC form.
static void export_csc(const Plan &P, const Numeric &F, cudaStream_t s,
                       std::vector<int64_t> &Lp, std::vector<int64_t> &Li,
                       std::vector<float> &Lx, std::vector<float> &D,
                       std::vector<float> &Dinv) {
  const Symbolic    &S = P.S;
  std::vector<float> pan(S.panel_elems);
  D.resize(S.n);
  Dinv.resize(S.n);
  if (S.panel_elems)
    MPIR_CUDA(cudaMemcpyAsync(pan.data(), F.panel.as<void>(), S.panel_elems * sizeof(float),
                              cudaMemcpyDeviceToHost, s));
  if (S.n) {
    MPIR_CUDA(cudaMemcpyAsync(D.data(), F.D.as<void>(), S.n * sizeof(float),
                              cudaMemcpyDeviceToHost, s));
    MPIR_CUDA(cudaMemcpyAsync(Dinv.data(), F.Dinv.as<void>(), S.n * sizeof(float),
                              cudaMemcpyDeviceToHost, s));
  }
  MPIR_CUDA(cudaStreamSynchronize(s));
  exact_pattern(S, Lp, Li);
  Lx.resize(Li.size());
  for (int64_t J = 0; J < S.ns; J++) {
    const int64_t f = S.sfirst[J], l = S.sfirst[J + 1], h = S.h(J);
    for (int64_t j = f; j < l; j++)
      for (int64_t p = Lp[j]; p < Lp[j + 1]; p++) {
        const int64_t lr = local_row(S, J, Li[p]);
        Lx[p] = lr < 0 ? 0.0f : pan[S.slofs[J] + (j - f) * h + lr];
      }
  }
}

// The leading k x k block of the factor in QDLDL's CSC form (columns < k,
// rows < k): row k' of L depends only on rows < k', so the pattern is the
// row-reach walk of rows < k, and only the panels of the supernodes holding
// columns < k are copied back.
static void export_csc_leading(const Plan &P, const Numeric &F, cudaStream_t s, int64_t k,
                               std::vector<int64_t> &Lp, std::vector<int64_t> &Li,
                               std::vector<float> &Lx, std::vector<float> &D) {
  const Symbolic &S = P.S;
  k = std::min<int64_t>(std::max<int64_t>(k, 0), S.n);
  // supernodes up to the one holding column k - 1
  int64_t Jend = 0;
  while (Jend < S.ns && S.sfirst[Jend] < k) Jend++;
  const int64_t npan = Jend > 0 ? S.slofs[Jend - 1] + S.w(Jend - 1) * S.h(Jend - 1) : 0;
  std::vector<float> pan(npan);
  D.resize(k);
  if (npan)
    MPIR_CUDA(cudaMemcpyAsync(pan.data(), F.panel.as<void>(), npan * sizeof(float),
                              cudaMemcpyDeviceToHost, s));
  if (k)
    MPIR_CUDA(cudaMemcpyAsync(D.data(), F.D.as<void>(), k * sizeof(float), cudaMemcpyDeviceToHost,
                              s));
  MPIR_CUDA(cudaStreamSynchronize(s));
  // column counts of the leading block: entries of rows < k
  std::vector<int64_t> cnt(k + 1, 0), mark(k, -1);
  for (int64_t r = 0; r < k; r++) {
    mark[r] = r;
    for (int64_t p = S.Cp[r]; p < S.Cp[r + 1]; p++)
      for (int64_t i = S.Ci[p]; mark[i] != r; i = S.etree[i]) {
        cnt[i + 1]++;
        mark[i] = r;
      }
  }
  Lp.assign(k + 1, 0);
  for (int64_t j = 0; j < k; j++) Lp[j + 1] = Lp[j] + cnt[j + 1];
  Li.resize(Lp[k]);
  std::vector<int64_t> next(Lp.begin(), Lp.end() - 1);
  std::fill(mark.begin(), mark.end(), -1);
  for (int64_t r = 0; r < k; r++) {
    mark[r] = r;
    for (int64_t p = S.Cp[r]; p < S.Cp[r + 1]; p++)
      for (int64_t i = S.Ci[p]; mark[i] != r; i = S.etree[i]) {
        Li[next[i]++] = r;
        mark[i]       = r;
      }
  }
  Lx.resize(Li.size());
  for (int64_t J = 0; J < Jend; J++) {
    const int64_t f = S.sfirst[J], l = std::min<int64_t>(S.sfirst[J + 1], k), h = S.h(J);
    for (int64_t j = f; j < l; j++)
      for (int64_t p = Lp[j]; p < Lp[j + 1]; p++) {
        const int64_t lr = local_row(S, J, Li[p]);
        Lx[p] = lr < 0 ? 0.0f : pan[S.slofs[J] + (j - f) * h + lr];
      }
  }
}

__global__ void k_f32_to_16(int64_t n, const float *in, uint16_t *out, int bf) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (bf) {
    const __nv_bfloat16 v = __float2bfloat16_rn(in[i]);
    out[i]                = *reinterpret_cast<const uint16_t *>(&v);
  } else {
    const __half v = __float2half_rn(in[i]);
    out[i]         = *reinterpret_cast<const uint16_t *>(&v);
  }
}

__global__ void k_16_to_f32(int64_t n, const uint16_t *in, float *out, int bf) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint16_t b = in[i];
  out[i] = bf ? __bfloat162float(*reinterpret_cast<const __nv_bfloat16 *>(&b))
              : __half2float(*reinterpret_cast<const __half *>(&b));
}

// Round float32 host data to a 16-bit type through the device's conversions.
static void to_16(const std::vector<float> &in, void *out, int prec, cudaStream_t s) {
  const int64_t n = static_cast<int64_t>(in.size());
  if (!n) return;
  DeviceBuffer a(n * sizeof(float)), b(n * sizeof(uint16_t));
  MPIR_CUDA(cudaMemcpyAsync(a.as<void>(), in.data(), n * sizeof(float), cudaMemcpyHostToDevice, s));
  launch(k_f32_to_16, static_cast<unsigned>((n + 255) / 256), 256, 0, s, 
      n, a.as<float>(), b.as<uint16_t>(), prec == kBF16);
  MPIR_CUDA(cudaMemcpyAsync(out, b.as<void>(), n * sizeof(uint16_t), cudaMemcpyDeviceToHost, s));
  MPIR_CUDA(cudaStreamSynchronize(s));
}

static void from_16(const void *in, int64_t n, int prec, std::vector<float> &out,
                    cudaStream_t s) {
  out.resize(n);
  if (!n) return;
  DeviceBuffer a(n * sizeof(uint16_t)), b(n * sizeof(float));
  MPIR_CUDA(cudaMemcpyAsync(a.as<void>(), in, n * sizeof(uint16_t), cudaMemcpyHostToDevice, s));
  launch(k_16_to_f32, static_cast<unsigned>((n + 255) / 256), 256, 0, s, 
      n, a.as<uint16_t>(), b.as<float>(), prec == kBF16);
  MPIR_CUDA(cudaMemcpyAsync(out.data(), b.as<void>(), n * sizeof(float), cudaMemcpyDeviceToHost, s));
  MPIR_CUDA(cudaStreamSynchronize(s));
}

struct StreamGuard {
  cudaStream_t s = nullptr;
  explicit StreamGuard(int device) {
    MPIR_CUDA(cudaSetDevice(device));
    MPIR_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  }
  ~StreamGuard() {
    if (s) {
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
  }
};

void invert_diag_blocks(const Plan &P, Numeric &F, cudaStream_t s);

}  // namespace mpir

using namespace mpir;

struct mpir_solver_s {
  Solver     *impl;
  std::string pending_log;  // rendered log awaiting mpir_solver_dump_log's copy
};

extern "C" {

int mpir_version(void) { return 10000; }

const char *mpir_last_error(void) { return g_err.c_str(); }

int mpir_device_count(int *count) {
  return guard([&]() -> int {
    int c = 0;
    MPIR_CUDA(cudaGetDeviceCount(&c));
    if (count) *count = c;
    return MPIR_OK;
  });
}

int64_t mpir_qdldl_etree(int64_t n, const int64_t *Ap, const int64_t *Ai, int64_t *work,
                         int64_t *Lnz, int64_t *etree) {
  return guard([&]() -> int64_t {
    if (n < 0 || (n > 0 && (!Ap || !Ai || !Lnz || !etree))) return MPIR_ERR_ARGUMENT;
    for (int64_t i = 0; i < n; i++) {
      if (work) work[i] = 0;
      Lnz[i]   = 0;
      etree[i] = -1;
    }
    return etree_counts(n, Ap, Ai, etree, Lnz);
  });
}

int64_t mpir_qdldl_factor(int64_t n, const int64_t *Ap, const int64_t *Ai, const double *Ax,
                          int64_t *Lp, int64_t *Li, void *Lx, void *D, void *Dinv,
                          int fact_prec, const int64_t *Lnz, const int64_t *etree,
                          int device) {
  return guard([&]() -> int64_t {
    if (fact_prec != kF32 && fact_prec != kBF16 && fact_prec != kF16)
      throw StatusError(MPIR_ERR_UNSUPPORTED, "factor type not provided (F32, BF16, F16)");
    if (n < 0) return MPIR_ERR_ARGUMENT;
    if (n == 0) {
      if (Lp) Lp[0] = 0;
      return 0;
    }
    Symbolic    S;
    std::string err;
    const int   rc = analyze(n, Ap, Ai, nullptr, Ordering::Natural, S, err);
    if (rc != kOk) throw StatusError(rc, err);
    for (int64_t j = 0; j < n; j++)
      if ((Lnz && Lnz[j] != S.Lnz[j]) || (etree && etree[j] != S.etree[j]))
        throw StatusError(MPIR_ERR_ARGUMENT, "Lnz / etree are not QDLDL_etree's output");
    StreamGuard sg(device);
    Plan        P;
    P.build(std::move(S), sg.s);
    Numeric F;
    F.allocate(P);
    MPIR_CUDA(cudaMemcpyAsync(F.Ax.as<void>(), Ax, P.S.nnz * sizeof(double),
                              cudaMemcpyHostToDevice, sg.s));
    // QDLDL_factor does not scale: an infinite threshold keeps AD = 1.
    F.run(P, F.Ax.as<double>(), std::numeric_limits<double>::infinity(), sg.s);
    const int64_t npos = F.result(sg.s);
    std::vector<int64_t> lp, li;
    std::vector<float>   lx, d, dinv;
    export_csc(P, F, sg.s, lp, li, lx, d, dinv);
    std::memcpy(Lp, lp.data(), (n + 1) * sizeof(int64_t));
    if (!li.empty()) std::memcpy(Li, li.data(), li.size() * sizeof(int64_t));
    if (fact_prec == kF32) {
      if (!lx.empty()) std::memcpy(Lx, lx.data(), lx.size() * sizeof(float));
      std::memcpy(D, d.data(), n * sizeof(float));
      std::memcpy(Dinv, dinv.data(), n * sizeof(float));
    } else {
      to_16(lx, Lx, fact_prec, sg.s);
      to_16(d, D, fact_prec, sg.s);
      to_16(dinv, Dinv, fact_prec, sg.s);
    }
    return npos;
  });
}

// The analysed, uploaded form of a caller's QDLDL factor, kept between
// QDLDL_solve calls: the reference's usage (LUIR_QDLDL, luir.hpp:165-205)
// solves with one factor many times, and the analysis of L's pattern, the
// packing into panels, the upload and the inversion of the diagonal blocks
// are then done once.  An entry is found by the device, the factor type and
// hashes of the whole of Lp, Li, Lx and Dinv (a factor rewritten in place
// misses the cache); the two most recently used entries are kept.
struct QdldlCached {
  int                             device = 0, prec = 0;
  int64_t                         n = 0;
  uint64_t                        hash = 0;
  std::unique_ptr<Plan>           P;
  std::unique_ptr<Numeric>        F;
  std::unique_ptr<SolveWorkspace> ws;
  DeviceBuffer                    xd;
  cudaStream_t                    s = nullptr;
  ~QdldlCached() {
    if (s) {
      cudaSetDevice(device);
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
  }
};
static std::mutex                               g_qdldl_mu;
static std::vector<std::unique_ptr<QdldlCached>> g_qdldl_cache;  // most recent last

static uint64_t hash_words(const void *p, size_t bytes, uint64_t h) {
  const unsigned char *c = static_cast<const unsigned char *>(p);
  size_t               i = 0;
  for (; i + 8 <= bytes; i += 8) {
    uint64_t w;
    std::memcpy(&w, c + i, 8);
    h = (h ^ w) * 0x100000001b3ull;
    h ^= h >> 29;
  }
  for (; i < bytes; i++) h = (h ^ c[i]) * 0x100000001b3ull;
  return h;
}

static int qdldl_solve_phases(int64_t n, const int64_t *Lp, const int64_t *Li, const void *Lx,
                              const void *Dinv, int fact_prec, void *x, int x_prec, int device,
                              int phases) {
  return guard([&]() -> int {
    if (fact_prec != kF32 && fact_prec != kBF16 && fact_prec != kF16)
      throw StatusError(MPIR_ERR_UNSUPPORTED, "factor type not provided (F32, BF16, F16)");
    if (x_prec != kF64 && x_prec != kF32)
      throw StatusError(MPIR_ERR_UNSUPPORTED, "vector type not provided (F64, F32)");
    if (n <= 0) return n < 0 ? MPIR_ERR_ARGUMENT : MPIR_OK;
    const int64_t nl    = Lp[n];
    const size_t  esize = fact_prec == kF32 ? 4 : 2;
    uint64_t      h     = 0xcbf29ce484222325ull ^ static_cast<uint64_t>(n);
    h = hash_words(Lp, (n + 1) * sizeof(int64_t), h);
    h = hash_words(Li, nl * sizeof(int64_t), h);
    h = hash_words(Lx, nl * esize, h);
    h = Dinv ? hash_words(Dinv, n * esize, h) : (h ^ 0x5bd1e995ull);
    std::lock_guard<std::mutex> lock(g_qdldl_mu);
    QdldlCached *E = nullptr;
    for (size_t i = 0; i < g_qdldl_cache.size(); i++) {
      QdldlCached &c = *g_qdldl_cache[i];
      if (c.device == device && c.prec == fact_prec && c.n == n && c.hash == h) {
        std::unique_ptr<QdldlCached> keep = std::move(g_qdldl_cache[i]);
        g_qdldl_cache.erase(g_qdldl_cache.begin() + i);
        g_qdldl_cache.push_back(std::move(keep));
        E = g_qdldl_cache.back().get();
        break;
      }
    }
    if (!E) {
      Symbolic    S;
      std::string err;
      const int   rc = analyze_from_L(n, Lp, Li, S, err);
      if (rc != kOk) throw StatusError(rc, err);
      auto c    = std::make_unique<QdldlCached>();
      c->device = device;
      c->prec   = fact_prec;
      c->n      = n;
      c->hash   = h;
      MPIR_CUDA(cudaSetDevice(device));
      MPIR_CUDA(cudaStreamCreateWithFlags(&c->s, cudaStreamNonBlocking));
      c->P = std::make_unique<Plan>();
      c->P->build(std::move(S), c->s);
      const Symbolic &Sy = c->P->S;
      c->F = std::make_unique<Numeric>();
      c->F->allocate(*c->P);
      std::vector<float> lx, dv(n, 1.0f);
      if (fact_prec == kF32) {
        lx.assign(static_cast<const float *>(Lx), static_cast<const float *>(Lx) + nl);
        if (Dinv) dv.assign(static_cast<const float *>(Dinv), static_cast<const float *>(Dinv) + n);
      } else {
        from_16(Lx, nl, fact_prec, lx, c->s);
        if (Dinv) from_16(Dinv, n, fact_prec, dv, c->s);
      }
      std::vector<float> pan(Sy.panel_elems, 0.0f);
      for (int64_t J = 0; J < Sy.ns; J++) {
        const int64_t f = Sy.sfirst[J], l = Sy.sfirst[J + 1], hh = Sy.h(J);
        for (int64_t j = f; j < l; j++) {
          pan[Sy.slofs[J] + (j - f) * hh + (j - f)] = 1.0f;
          for (int64_t p = Lp[j]; p < Lp[j + 1]; p++)
            pan[Sy.slofs[J] + (j - f) * hh + local_row(Sy, J, Li[p])] = lx[p];
        }
      }
      MPIR_CUDA(cudaMemcpyAsync(c->F->panel.as<void>(), pan.data(), pan.size() * sizeof(float),
                                cudaMemcpyHostToDevice, c->s));
      MPIR_CUDA(cudaMemcpyAsync(c->F->Dinv.as<void>(), dv.data(), n * sizeof(float),
                                cudaMemcpyHostToDevice, c->s));
      invert_diag_blocks(*c->P, *c->F, c->s);
      c->F->trim();  // the solves read L, Dinv and the block inverses only
      c->ws = std::make_unique<SolveWorkspace>();
      c->ws->allocate(*c->P);
      c->xd.resize(n * sizeof(double));
      MPIR_CUDA(cudaStreamSynchronize(c->s));
      if (g_qdldl_cache.size() >= 2) g_qdldl_cache.erase(g_qdldl_cache.begin());
      g_qdldl_cache.push_back(std::move(c));
      E = g_qdldl_cache.back().get();
    }
    MPIR_CUDA(cudaSetDevice(device));
    std::vector<double> xh(n);
    for (int64_t i = 0; i < n; i++)
      xh[i] = x_prec == kF64 ? static_cast<const double *>(x)[i]
                             : static_cast<double>(static_cast<const float *>(x)[i]);
    MPIR_CUDA(cudaMemcpyAsync(E->xd.as<void>(), xh.data(), n * sizeof(double),
                              cudaMemcpyHostToDevice, E->s));
    ldlt_solve(*E->P, *E->F, E->xd.as<double>(), *E->ws, E->s, phases);
    MPIR_CUDA(cudaMemcpyAsync(xh.data(), E->xd.as<void>(), n * sizeof(double),
                              cudaMemcpyDeviceToHost, E->s));
    MPIR_CUDA(cudaStreamSynchronize(E->s));
    int32_t wait_err = 0;
    MPIR_CUDA(cudaMemcpy(&wait_err, E->ws->err.as<void>(), sizeof wait_err, cudaMemcpyDeviceToHost));
    if (wait_err != 0) {
      device_zero(E->ws->err.as<void>(), sizeof wait_err);
      g_err = "a bounded device wait of the triangular solves ran out";
      return MPIR_ERR_TIMEOUT;
    }
    for (int64_t i = 0; i < n; i++) {
      if (x_prec == kF64)
        static_cast<double *>(x)[i] = xh[i];
      else
        static_cast<float *>(x)[i] = static_cast<float>(xh[i]);
    }
    return MPIR_OK;
  });
}

int mpir_qdldl_solve(int64_t n, const int64_t *Lp, const int64_t *Li, const void *Lx,
                     const void *Dinv, int fact_prec, void *x, int x_prec, int device) {
  return qdldl_solve_phases(n, Lp, Li, Lx, Dinv, fact_prec, x, x_prec, device, kAllPhases);
}

int mpir_qdldl_lsolve(int64_t n, const int64_t *Lp, const int64_t *Li, const void *Lx,
                      int fact_prec, void *x, int x_prec, int device) {
  return qdldl_solve_phases(n, Lp, Li, Lx, nullptr, fact_prec, x, x_prec, device, kForward);
}

int mpir_qdldl_ltsolve(int64_t n, const int64_t *Lp, const int64_t *Li, const void *Lx,
                       int fact_prec, void *x, int x_prec, int device) {
  return qdldl_solve_phases(n, Lp, Li, Lx, nullptr, fact_prec, x, x_prec, device, kBackward);
}

int mpir_qdldl_solve_noalloc(int64_t n, const int64_t *Lp, const int64_t *Li, const float *Lx,
                             const float *Dinv, double *x, int device) {
  return guard([&]() -> int {
    if (n > 0 && (!Lp || !Li || !Lx || !Dinv || !x)) return MPIR_ERR_ARGUMENT;
    std::string err;
    const int   rc = qdldl_solve_noalloc(n, Lp, Li, Lx, Dinv, x, device, err);
    if (rc != MPIR_OK) throw StatusError(rc, err);
    return MPIR_OK;
  });
}

int mpir_solver_create(mpir_solver *out, int uf, int uw, int ur, int device) {
  return guard([&]() -> int {
    if (!out) return MPIR_ERR_ARGUMENT;
    *out = nullptr;
    if ((uf != kF64 && uf != kF32 && uf != kBF16 && uf != kF16) || uw != kF64 ||
        (ur != kF64 && ur != kDD))
      throw StatusError(MPIR_ERR_UNSUPPORTED,
                        "provided precisions: UF=F64/F32/BF16/F16, UW=F64, UR=F64 or DD");
    auto *h = new mpir_solver_s{nullptr, {}};
    try {
      h->impl = new Solver(uf, uw, ur, device);
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
    return MPIR_OK;
  });
}

int mpir_solver_destroy(mpir_solver s) {
  return guard([&]() -> int {
    if (s) {
      delete s->impl;
      delete s;
    }
    return MPIR_OK;
  });
}

#define MPIR_NEED(s)                                          \
  if (!(s) || !(s)->impl) {                                   \
    g_err = "null solver handle";                             \
    return MPIR_ERR_ARGUMENT;                                 \
  }

int mpir_solver_set_max_ir_iterations(mpir_solver s, int64_t n) {
  MPIR_NEED(s);
  if (n < 0) return MPIR_ERR_ARGUMENT;
  s->impl->ir_iter = n;
  return MPIR_OK;
}
int mpir_solver_set_max_gmres_iterations(mpir_solver s, int64_t n) {
  MPIR_NEED(s);
  if (n < 0) return MPIR_ERR_ARGUMENT;
  s->impl->gmres_iter = n;
  return MPIR_OK;
}
int mpir_solver_set_tolerance(mpir_solver s, double tol) {
  MPIR_NEED(s);
  s->impl->tol = tol;
  return MPIR_OK;
}

int mpir_solver_analyze(mpir_solver s, int64_t n, const int64_t *Ap, const int64_t *Ai,
                        const double *Ax, int ordering) {
  MPIR_NEED(s);
  return guard([&]() -> int {
    if (n < 0 || (n > 0 && (!Ap || !Ai))) return MPIR_ERR_ARGUMENT;
    if (ordering != MPIR_ORDER_NATURAL && ordering != MPIR_ORDER_AUTO) return MPIR_ERR_ARGUMENT;
    Symbolic    probe;
    std::string err;
    // Input errors surface with QDLDL's codes before anything is allocated.
    for (int64_t j = 0; j < n; j++) {
      if (Ap[j] == Ap[j + 1]) throw StatusError(MPIR_ERR_INPUT, "empty column " + std::to_string(j));
      for (int64_t p = Ap[j]; p < Ap[j + 1]; p++)
        if (Ai[p] > j || Ai[p] < 0)
          throw StatusError(MPIR_ERR_INPUT, "entry below the diagonal in column " + std::to_string(j));
    }
    return s->impl->analyze(n, Ap, Ai, Ax, ordering);
  });
}

int mpir_solver_factor(mpir_solver s, const double *Ax) {
  MPIR_NEED(s);
  return guard([&]() -> int {
    const int rc = s->impl->factor(Ax);
    if (rc == kBadInput) g_err = "zero pivot";
    if (rc == MPIR_ERR_TIMEOUT) g_err = "a bounded device wait ran out";
    return rc;
  });
}

int mpir_solver_factor_device(mpir_solver s, const double *d_Ax) {
  MPIR_NEED(s);
  return guard([&]() -> int {
    const int rc = s->impl->factor_device(d_Ax);
    if (rc == kBadInput) g_err = "zero pivot";
    if (rc == MPIR_ERR_TIMEOUT) g_err = "a bounded device wait ran out";
    return rc;
  });
}

int mpir_solver_compute(mpir_solver s, int64_t n, const int64_t *Ap, const int64_t *Ai,
                        const double *Ax) {
  const int rc = mpir_solver_analyze(s, n, Ap, Ai, Ax, MPIR_ORDER_AUTO);
  if (rc != MPIR_OK) return rc;
  return mpir_solver_factor(s, Ax);
}

int mpir_solver_solve(mpir_solver s, const double *b, double *x, mpir_report *rep) {
  MPIR_NEED(s);
  static_assert(sizeof(mpir_report) == sizeof(Report), "report layout");
  return guard([&]() -> int {
    return s->impl->solve(b, x, reinterpret_cast<Report *>(rep));
  });
}

int mpir_solver_solve_device(mpir_solver s, const double *d_b, double *d_x, mpir_report *rep) {
  MPIR_NEED(s);
  return guard([&]() -> int {
    return s->impl->solve_device(d_b, d_x, reinterpret_cast<Report *>(rep));
  });
}

int mpir_solver_solve_many(mpir_solver s, int64_t nrhs, const double *B, double *X,
                           mpir_report *reps) {
  MPIR_NEED(s);
  return guard([&]() -> int {
    if (nrhs < 0 || (nrhs > 0 && (!B || !X)))
      throw StatusError(MPIR_ERR_ARGUMENT, "invalid argument");
    const int64_t n  = s->impl->plan().S.n;
    const int64_t mb = Solver::kMaxBatch;
    for (int64_t k0 = 0; k0 < nrhs; k0 += mb) {
      const int nb = static_cast<int>(std::min(mb, nrhs - k0));
      Report   *r  = reps ? reinterpret_cast<Report *>(reps + k0) : nullptr;
      const int rc = nb == 1 ? s->impl->solve(B + k0 * n, X + k0 * n, r)
                             : s->impl->solve_batch(nb, B + k0 * n, X + k0 * n, r);
      if (rc != MPIR_OK) return rc;
    }
    return MPIR_OK;
  });
}

int mpir_solver_solve_batch(mpir_solver s, int nrhs, const double *B, double *X,
                            mpir_report *reps) {
  MPIR_NEED(s);
  return guard([&]() -> int {
    if (nrhs < 1 || nrhs > Solver::kMaxBatch || !B || !X)
      throw StatusError(MPIR_ERR_ARGUMENT, "1 <= nrhs <= 16 right-hand sides, non-NULL B and X");
    return s->impl->solve_batch(nrhs, B, X, reinterpret_cast<Report *>(reps));
  });
}

int mpir_solver_solve_batch_device(mpir_solver s, int nrhs, const double *d_B, double *d_X,
                                   mpir_report *reps) {
  MPIR_NEED(s);
  return guard([&]() -> int {
    if (nrhs < 1 || nrhs > Solver::kMaxBatch || !d_B || !d_X)
      throw StatusError(MPIR_ERR_ARGUMENT, "1 <= nrhs <= 16 right-hand sides, non-NULL B and X");
    return s->impl->solve_batch_device(nrhs, d_B, d_X, reinterpret_cast<Report *>(reps));
  });
}

int mpir_solver_apply_factor(mpir_solver s, int nrhs, double *X) {
  MPIR_NEED(s);
  return guard([&]() -> int {
    if (nrhs < 1 || nrhs > Solver::kMaxBatch || !X)
      throw StatusError(MPIR_ERR_ARGUMENT, "1 <= nrhs <= 16 vectors, non-NULL X");
    Solver       &sv = *s->impl;
    const int64_t n  = sv.plan().S.n;
    if (n == 0) return MPIR_OK;
    DeviceBuffer d(n * nrhs * sizeof(double));
    MPIR_CUDA(cudaMemcpyAsync(d.as<void>(), X, n * nrhs * sizeof(double), cudaMemcpyHostToDevice,
                              sv.stream()));
    sv.precond_device(nrhs, d.as<double>());
    MPIR_CUDA(cudaMemcpyAsync(X, d.as<void>(), n * nrhs * sizeof(double), cudaMemcpyDeviceToHost,
                              sv.stream()));
    MPIR_CUDA(cudaStreamSynchronize(sv.stream()));
    return MPIR_OK;
  });
}

int mpir_solver_set_wait_controls(mpir_solver s, int poll_log2, int withhold_item) {
  MPIR_NEED(s);
  return guard([&]() -> int {
    if (poll_log2 < 0 || poll_log2 > 30)
      throw StatusError(MPIR_ERR_ARGUMENT, "poll_log2 in 0 .. 30");
    s->impl->set_wait_controls(poll_log2, withhold_item);
    return MPIR_OK;
  });
}

int mpir_solver_dump_log(mpir_solver s, char *buf, int64_t cap, int64_t *len) {
  MPIR_NEED(s);
  return guard([&]() -> int {
    if (!len) throw StatusError(MPIR_ERR_ARGUMENT, "len is NULL");
    if (s->pending_log.empty()) s->pending_log = s->impl->dump_log();
    *len = static_cast<int64_t>(s->pending_log.size()) + 1;
    if (!buf || cap < *len) return MPIR_OK;
    std::memcpy(buf, s->pending_log.c_str(), static_cast<size_t>(*len));
    s->pending_log.clear();
    return MPIR_OK;
  });
}

int mpir_solver_luir(mpir_solver s, const double *b, double *x, int maxiter, mpir_report *rep) {
  MPIR_NEED(s);
  return guard([&]() -> int {
    if (maxiter < 0) throw StatusError(MPIR_ERR_ARGUMENT, "maxiter must be >= 0");
    return s->impl->luir(b, x, maxiter, reinterpret_cast<Report *>(rep));
  });
}

int mpir_solver_residual(mpir_solver s, const double *b, const double *x, double *r,
                         int res_prec, double *rinf) {
  MPIR_NEED(s);
  return guard([&]() -> int {
    if (res_prec != MPIR_F64 && res_prec != MPIR_DD)
      throw StatusError(MPIR_ERR_ARGUMENT, "res_prec must be MPIR_F64 or MPIR_DD");
    if (s->impl->analyzed() && s->impl->plan().S.n > 0 && (!b || !x || !r))
      throw StatusError(MPIR_ERR_ARGUMENT, "invalid argument");
    const double m = s->impl->residual(b, x, r, res_prec == MPIR_DD);
    if (rinf) *rinf = m;
    return MPIR_OK;
  });
}

int mpir_solver_luir_device(mpir_solver s, const double *d_b, double *d_x, int maxiter,
                            mpir_report *rep) {
  MPIR_NEED(s);
  return guard([&]() -> int {
    if (maxiter < 0) throw StatusError(MPIR_ERR_ARGUMENT, "maxiter must be >= 0");
    return s->impl->luir_device(d_b, d_x, maxiter, reinterpret_cast<Report *>(rep));
  });
}

int mpir_luir_qdldl(int64_t n, const int64_t *Ap, const int64_t *Ai, const double *Ax,
                    const double *b, double *x, int fact_prec, int maxiter, mpir_report *rep,
                    int device) {
  return guard([&]() -> int {
    if (n < 0 || !Ap || !Ai || !Ax || !b || !x || maxiter < 0)
      throw StatusError(MPIR_ERR_ARGUMENT, "invalid argument");
    if (fact_prec != kF32 && fact_prec != kBF16 && fact_prec != kF16)
      throw StatusError(MPIR_ERR_UNSUPPORTED, "provided factor types: F32, BF16, F16");
    for (int64_t j = 0; j < n; j++) {
      if (Ap[j + 1] <= Ap[j])
        throw StatusError(MPIR_ERR_INPUT, "empty column " + std::to_string(j));
      for (int64_t p = Ap[j]; p < Ap[j + 1]; p++)
        if (Ai[p] > j)
          throw StatusError(MPIR_ERR_INPUT, "entry below the diagonal in column " + std::to_string(j));
    }
    Solver sv(fact_prec, kF64, kF64, device);
    sv.analyze(n, Ap, Ai, Ax, MPIR_ORDER_AUTO);
    const int fr = sv.factor(Ax);
    if (fr == kBadInput) {
      g_err = "zero pivot";
      return fr;
    }
    if (fr != kOk) return fr;
    return sv.luir(b, x, maxiter, reinterpret_cast<Report *>(rep));
  });
}

int mpir_solver_set_update(mpir_solver s, int engine) {
  MPIR_NEED(s);
  return guard([&]() -> int {
    s->impl->set_update_engine(engine);
    return MPIR_OK;
  });
}

int mpir_solver_set_stream(mpir_solver s, void *stream) {
  MPIR_NEED(s);
  s->impl->set_stream(static_cast<cudaStream_t>(stream));
  return MPIR_OK;
}

int mpir_solver_info(mpir_solver s, mpir_info *info) {
  MPIR_NEED(s);
  return guard([&]() -> int {
    if (!info) return MPIR_ERR_ARGUMENT;
    std::memset(info, 0, sizeof *info);
    const Solver &sv = *s->impl;
    const Plan   &P  = sv.plan();
    const Symbolic &S = P.S;
    info->n            = S.n;
    info->nnz_upper    = S.nnz;
    info->nnz_L        = S.nnzL;
    info->supernodes   = S.ns;
    info->levels       = S.nlevels;
    info->panel_bytes  = S.panel_elems * 4;
    info->update_bytes = S.uarena_elems * 4;
    info->max_front    = S.max_h;
    double fl = 0;
    for (int64_t j = 0; j < S.n; j++) fl += static_cast<double>(S.Lnz[j]) * S.Lnz[j];
    info->factor_flops     = fl;
    info->solve_bytes      = 2.0 * 4.0 * S.nnzL + 4.0 * S.n + 4.0 * 8.0 * S.n;
    info->update_flops     = P.update_flops;
    info->trsm_flops       = P.trsm_flops;
    info->panel_read_bytes = P.panel_read_bytes;
    return MPIR_OK;
  });
}

int mpir_solver_symbolic(mpir_solver s, int64_t *perm, int64_t *etree, int64_t *Lnz,
                         int64_t *Cp, int64_t *Ci, int64_t *Csrc) {
  MPIR_NEED(s);
  return guard([&]() -> int {
    const Symbolic &S = s->impl->plan().S;
    auto put = [](int64_t *dst, const std::vector<int64_t> &v) {
      if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(int64_t));
    };
    put(perm, S.perm);
    put(etree, S.etree);
    put(Lnz, S.Lnz);
    put(Cp, S.Cp);
    put(Ci, S.Ci);
    put(Csrc, S.Csrc);
    return MPIR_OK;
  });
}

int mpir_solver_supernodes(mpir_solver s, int64_t *sfirst, int64_t *srowptr, int32_t *srows,
                           int64_t *nrows) {
  MPIR_NEED(s);
  return guard([&]() -> int {
    const Symbolic &S = s->impl->plan().S;
    if (sfirst) std::memcpy(sfirst, S.sfirst.data(), S.sfirst.size() * sizeof(int64_t));
    if (srowptr) std::memcpy(srowptr, S.srowptr.data(), S.srowptr.size() * sizeof(int64_t));
    if (srows && !S.srows.empty())
      std::memcpy(srows, S.srows.data(), S.srows.size() * sizeof(int32_t));
    if (nrows) *nrows = static_cast<int64_t>(S.srows.size());
    return MPIR_OK;
  });
}

int mpir_solver_export_factor(mpir_solver s, int64_t *Lp, int64_t *Li, float *Lx, float *D,
                              float *Dinv) {
  MPIR_NEED(s);
  return guard([&]() -> int {
    const Solver &sv = *s->impl;
    if (!sv.numeric().valid) throw std::logic_error("no valid factor");
    std::vector<int64_t> lp, li;
    std::vector<float>   lx, d, dinv;
    export_csc(sv.plan(), sv.numeric(), sv.stream(), lp, li, lx, d, dinv);
    const int64_t n = sv.plan().S.n;
    if (Lp) std::memcpy(Lp, lp.data(), (n + 1) * sizeof(int64_t));
    if (Li && !li.empty()) std::memcpy(Li, li.data(), li.size() * sizeof(int64_t));
    if (Lx && !lx.empty()) std::memcpy(Lx, lx.data(), lx.size() * sizeof(float));
    if (D && n) std::memcpy(D, d.data(), n * sizeof(float));
    if (Dinv && n) std::memcpy(Dinv, dinv.data(), n * sizeof(float));
    return MPIR_OK;
  });
}

int mpir_solver_export_factor_leading(mpir_solver s, int64_t k, int64_t *Lp, int64_t *Li,
                                      float *Lx, float *D, int64_t *nnz) {
  MPIR_NEED(s);
  return guard([&]() -> int {
    const Solver &sv = *s->impl;
    if (!sv.numeric().valid) throw std::logic_error("no valid factor");
    if (k < 0 || k > sv.plan().S.n) throw StatusError(MPIR_ERR_ARGUMENT, "0 <= k <= n");
    std::vector<int64_t> lp, li;
    std::vector<float>   lx, d;
    export_csc_leading(sv.plan(), sv.numeric(), sv.stream(), k, lp, li, lx, d);
    if (nnz) *nnz = static_cast<int64_t>(li.size());
    if (Lp) std::memcpy(Lp, lp.data(), (k + 1) * sizeof(int64_t));
    if (Li && !li.empty()) std::memcpy(Li, li.data(), li.size() * sizeof(int64_t));
    if (Lx && !lx.empty()) std::memcpy(Lx, lx.data(), lx.size() * sizeof(float));
    if (D && k) std::memcpy(D, d.data(), k * sizeof(float));
    return MPIR_OK;
  });
}

int mpir_analyze_host(int64_t n, const int64_t *Ap, const int64_t *Ai, const double *Ax,
                      int ordering, int64_t *perm, int64_t *etree, int64_t *Lnz, int64_t *Cp,
                      int64_t *Ci, int64_t *Lp, int64_t *Li, mpir_info *info) {
  return guard([&]() -> int {
    if (n < 0 || (n > 0 && (!Ap || !Ai))) return MPIR_ERR_ARGUMENT;
    std::vector<int8_t> sign;
    if (Ax) {
      sign.assign(n, 0);
      for (int64_t j = 0; j < n; j++)
        for (int64_t p = Ap[j]; p < Ap[j + 1]; p++)
          if (Ai[p] == j && Ax[p] > 0) sign[j] = 1;
    }
    Symbolic    S;
    std::string err;
    const int   rc = analyze(n, Ap, Ai, Ax ? sign.data() : nullptr,
                             static_cast<Ordering>(ordering), S, err);
    if (rc != kOk) throw StatusError(rc, err);
    auto put = [](int64_t *dst, const std::vector<int64_t> &v) {
      if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(int64_t));
    };
    put(perm, S.perm);
    put(etree, S.etree);
    put(Lnz, S.Lnz);
    put(Cp, S.Cp);
    put(Ci, S.Ci);
    if (Lp || Li) {
      std::vector<int64_t> lp, li;
      exact_pattern(S, lp, li);
      put(Lp, lp);
      put(Li, li);
    }
    if (info) {
      std::memset(info, 0, sizeof *info);
      info->n            = S.n;
      info->nnz_upper    = S.nnz;
      info->nnz_L        = S.nnzL;
      info->supernodes   = S.ns;
      info->levels       = S.nlevels;
      info->panel_bytes  = S.panel_elems * 4;
      info->update_bytes = S.uarena_elems * 4;
      info->max_front    = S.max_h;
      double fl = 0;
      for (int64_t j = 0; j < S.n; j++) fl += static_cast<double>(S.Lnz[j]) * S.Lnz[j];
      info->factor_flops = fl;
      info->solve_bytes  = 2.0 * 4.0 * S.nnzL + 4.0 * S.n + 4.0 * 8.0 * S.n;
    }
    return MPIR_OK;
  });
}

struct mpir_group_s {
  FactorGroup *impl;
};

int mpir_group_create(mpir_group *out, mpir_solver s, int k) {
  MPIR_NEED(s);
  return guard([&]() -> int {
    if (!out || k < 1) throw StatusError(MPIR_ERR_ARGUMENT, "NULL output or k < 1");
    *out = nullptr;
    auto *g = new mpir_group_s{nullptr};
    try {
      g->impl = new FactorGroup(*s->impl, k);
    } catch (...) {
      delete g;
      throw;
    }
    *out = g;
    return MPIR_OK;
  });
}

int mpir_group_factor(mpir_group g, const double *Ax, int64_t *npos) {
  return guard([&]() -> int {
    if (!g || !g->impl || !Ax) throw StatusError(MPIR_ERR_ARGUMENT, "NULL argument");
    const int64_t nnz = g->impl->member(0).plan().S.nnz;
    const int     rc  = g->impl->factor(Ax, nnz, npos);
    if (rc == kBadInput) g_err = "zero pivot in a member of the group";
    if (rc == MPIR_ERR_TIMEOUT) g_err = "a bounded device wait ran out";
    return rc;
  });
}

int mpir_group_solve(mpir_group g, int member, const double *b, double *x, mpir_report *rep) {
  return guard([&]() -> int {
    if (!g || !g->impl || !b || !x) throw StatusError(MPIR_ERR_ARGUMENT, "NULL argument");
    if (member < 0 || member >= g->impl->size())
      throw StatusError(MPIR_ERR_ARGUMENT, "member out of range");
    return g->impl->member(member).solve(b, x, reinterpret_cast<Report *>(rep));
  });
}

int mpir_group_solve_batch(mpir_group g, int member, int nrhs, const double *B, double *X,
                           mpir_report *reps) {
  return guard([&]() -> int {
    if (!g || !g->impl || !B || !X) throw StatusError(MPIR_ERR_ARGUMENT, "NULL argument");
    if (member < 0 || member >= g->impl->size())
      throw StatusError(MPIR_ERR_ARGUMENT, "member out of range");
    if (nrhs < 1 || nrhs > Solver::kMaxBatch)
      throw StatusError(MPIR_ERR_ARGUMENT, "1 <= nrhs <= 16 right-hand sides");
    Solver &m = g->impl->member(member);
    return nrhs == 1 ? m.solve(B, X, reinterpret_cast<Report *>(reps))
                     : m.solve_batch(nrhs, B, X, reinterpret_cast<Report *>(reps));
  });
}

int mpir_group_destroy(mpir_group g) {
  return guard([&]() -> int {
    if (g) {
      delete g->impl;
      delete g;
    }
    return MPIR_OK;
  });
}

struct mpir_server_s {
  Server *impl;
};

int mpir_server_create(mpir_server *out, const mpir_server_config *cfg) {
  return guard([&]() -> int {
    if (!out || !cfg) throw StatusError(MPIR_ERR_ARGUMENT, "NULL argument");
    *out = nullptr;
    if ((cfg->uf != kF32 && cfg->uf != kBF16 && cfg->uf != kF16) ||
        (cfg->ur != kF64 && cfg->ur != kDD))
      throw StatusError(MPIR_ERR_UNSUPPORTED, "provided precisions: UF=F32/BF16/F16, UR=F64/DD");
    if (cfg->workers < 1 || cfg->max_batch < 1 || cfg->budget_bytes <= 0 ||
        cfg->max_ir_iterations < 0 || cfg->max_gmres_iterations < 0)
      throw StatusError(MPIR_ERR_ARGUMENT, "invalid server configuration");
    ServerConfig c;
    c.device               = cfg->device;
    c.uf                   = cfg->uf;
    c.ur                   = cfg->ur;
    c.workers              = cfg->workers;
    c.max_batch            = cfg->max_batch;
    if (cfg->update < 0 || cfg->update > 2)
      throw StatusError(MPIR_ERR_ARGUMENT, "update engine: 0 default, 1 3xTF32, 2 3xBF16");
    c.update               = cfg->update;
    c.budget_bytes         = cfg->budget_bytes;
    c.max_ir_iterations    = cfg->max_ir_iterations;
    c.max_gmres_iterations = cfg->max_gmres_iterations;
    c.tolerance            = cfg->tolerance;
    MPIR_CUDA(cudaSetDevice(c.device));
    *out = new mpir_server_s{new Server(c)};
    return MPIR_OK;
  });
}

int mpir_server_submit(mpir_server s, const mpir_server_request *r, int64_t *id) {
  return guard([&]() -> int {
    if (!s || !s->impl || !r || !id) throw StatusError(MPIR_ERR_ARGUMENT, "NULL argument");
    if (r->n < 0 || (r->n > 0 && (!r->Ap || !r->Ai || !r->Ax || !r->b || !r->x)))
      throw StatusError(MPIR_ERR_ARGUMENT, "request arrays missing");
    for (int64_t j = 0; j < r->n; j++) {
      if (r->Ap[j + 1] <= r->Ap[j])
        throw StatusError(MPIR_ERR_INPUT, "empty column " + std::to_string(j));
      if (r->Ai[r->Ap[j + 1] - 1] > j)
        throw StatusError(MPIR_ERR_INPUT, "entry below the diagonal in column " + std::to_string(j));
    }
    ServerRequest q;
    q.pattern_key = r->pattern_key;
    q.values_key  = r->values_key;
    q.n           = r->n;
    q.Ap          = r->Ap;
    q.Ai          = r->Ai;
    q.Ax          = r->Ax;
    q.b           = r->b;
    q.x           = r->x;
    *id           = s->impl->submit(q);
    return MPIR_OK;
  });
}

int mpir_server_wait(mpir_server s, int64_t id, mpir_server_result *res) {
  return guard([&]() -> int {
    if (!s || !s->impl) throw StatusError(MPIR_ERR_ARGUMENT, "NULL server");
    ServerResult r;
    s->impl->wait(id, &r);
    if (res) {
      std::memset(res, 0, sizeof *res);
      res->id         = r.id;
      res->status     = r.status;
      res->path       = r.path;
      res->batch      = r.batch;
      res->latency_ms = r.latency_ms;
      res->queue_ms   = r.queue_ms;
      res->service_ms = r.service_ms;
      static_assert(sizeof(mpir_report) == sizeof(Report), "report layout");
      std::memcpy(&res->report, &r.report, sizeof(Report));
    }
    if (r.status != 0) g_err = r.message;
    return MPIR_OK;
  });
}

int mpir_server_drain(mpir_server s) {
  return guard([&]() -> int {
    if (!s || !s->impl) throw StatusError(MPIR_ERR_ARGUMENT, "NULL server");
    s->impl->drain();
    return MPIR_OK;
  });
}

int mpir_server_get_stats(mpir_server s, mpir_server_stats *out) {
  return guard([&]() -> int {
    if (!s || !s->impl || !out) throw StatusError(MPIR_ERR_ARGUMENT, "NULL argument");
    const ServerStats st = s->impl->stats();
    out->submitted         = st.submitted;
    out->completed         = st.completed;
    out->failed            = st.failed;
    out->refused           = st.refused;
    out->analyses          = st.analyses;
    out->factorizations    = st.factorizations;
    out->solves            = st.solves;
    out->batched_solves    = st.batched_solves;
    out->batched_rhs       = st.batched_rhs;
    out->evictions         = st.evictions;
    out->resident_factors  = st.resident_factors;
    out->resident_patterns = st.resident_patterns;
    out->queued            = st.queued;
    out->bytes_in_use      = st.bytes_in_use;
    out->peak_bytes        = st.peak_bytes;
    out->analysis_reuses   = st.analysis_reuses;
    out->plan_uploads      = st.plan_uploads;
    out->analysis_ms       = st.analysis_ms;
    out->plan_ms           = st.plan_ms;
    out->factor_ms         = st.factor_ms;
    out->solve_ms          = st.solve_ms;
    out->factor_device_ms  = st.factor_device_ms;
    out->solve_device_ms   = st.solve_device_ms;
    out->setup_ms          = st.setup_ms;
    out->trim_ms           = st.trim_ms;
    out->plan_upload_ms    = st.plan_upload_ms;
    return MPIR_OK;
  });
}

int mpir_server_destroy(mpir_server s) {
  return guard([&]() -> int {
    if (s) {
      delete s->impl;
      delete s;
    }
    return MPIR_OK;
  });
}

int64_t mpir_launch_count(void) { return launch_total(); }

int mpir_kernel_timer_enable(int on) {
  KernelTimer &t = kernel_timer();
  t.enabled      = on != 0;
  t.reset();
  return MPIR_OK;
}

int mpir_kernel_timer_collect(double *ms, int64_t *launches, int nclass) {
  return guard([&]() -> int {
    MPIR_CUDA(cudaDeviceSynchronize());
    kernel_timer().collect(ms, launches, nclass);
    return MPIR_OK;
  });
}

}  // extern "C"
