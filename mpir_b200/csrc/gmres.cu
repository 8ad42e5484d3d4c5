// GMRES-IR on the device: GmresLDLIR::Solve (gmres_ir.hpp:536-634) and
// PrecondGmres (gmres_ir.hpp:636-741) with the supernodal LDL^T factor as the
// left preconditioner.  Vectors and the Arnoldi basis are float64 in the
// permuted order; the host keeps the small Hessenberg least-squares problem
// and its Givens rotations, reading back one column of H per inner step.
#include <cfloat>
#include <chrono>
#include <cstdio>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "solve_dev.cuh"
#include "solver.hpp"

namespace mpir {

double eps_of(int prec) {
  switch (prec) {
    case kF64: return DBL_EPSILON;
    case kF32: return FLT_EPSILON;
    case kBF16: return 0.0078125;          // 2^-7
    case kF16: return 0.0009765625;        // 2^-10
    case kDD: return 4.93038065763132e-32;  // 2^-104
  }
  return DBL_EPSILON;
}

// Trailing-update engine for a factor type: float32 runs 3xTF32 tensor-core
// products (float32-level accuracy), bfloat16 / float16 factors single-pass
// tensor-core products in that type; a float32 factor may instead take
// 3xBF16 products (about 16 significant bits, twice the 3xTF32 rate:
// Solver::update_engine = kUpdateBF16x3); MPIR_UPDATE ("simt" = float32 SIMT
// units, "tf32x3", "bf16x3", "bf16", "f16") overrides.
static int update_mode_for(int uf, int engine) {
  int mode = uf == kBF16 ? 0 : uf == kF16 ? 2 : engine == kUpdateBF16x3 ? 3 : 1;
  if (const char *e = std::getenv("MPIR_UPDATE")) {
    const std::string v(e);
    if (v == "simt") mode = -1;
    else if (v == "bf16") mode = 0;
    else if (v == "tf32x3") mode = 1;
    else if (v == "f16") mode = 2;
    else if (v == "bf16x3") mode = 3;
  }
  return mode;
}

Solver::Solver(int uf_, int uw_, int ur_, int dev)
    : device(dev), uf(uf_), uw(uw_), ur(ur_) {
  MPIR_CUDA(cudaSetDevice(device));
  MPIR_CUDA(cudaStreamCreateWithFlags(&own_stream_, cudaStreamNonBlocking));
  stream_ = own_stream_;
  MPIR_CUDA(cudaEventCreate(&ev0_));
  MPIR_CUDA(cudaEventCreate(&ev1_));
}

Solver::~Solver() {
  cudaSetDevice(device);
  if (own_stream_) cudaStreamSynchronize(own_stream_);
  if (stream_ && stream_ != own_stream_) cudaStreamSynchronize(stream_);
  if (hpin_) pinned_free(hpin_, hpin_bytes_);
  if (ev0_) cudaEventDestroy(ev0_);
  if (ev1_) cudaEventDestroy(ev1_);
  plan_.reset();
  if (own_stream_) cudaStreamDestroy(own_stream_);
}

int Solver::analyze(int64_t n, const int64_t *Ap, const int64_t *Ai,
                    const double *Ax, int ordering) {
  MPIR_CUDA(cudaSetDevice(device));
  std::vector<int8_t> sign;
  if (Ax) {
    sign.assign(n, 0);
    for (int64_t j = 0; j < n; j++)
      for (int64_t p = Ap[j]; p < Ap[j + 1]; p++)
        if (Ai[p] == j && Ax[p] > 0) sign[j] = 1;
  }
  Symbolic    S;
  std::string err;
  const int   rc = mpir::analyze(n, Ap, Ai, Ax ? sign.data() : nullptr,
                                 static_cast<Ordering>(ordering), S, err);
  if (rc != kOk) throw std::invalid_argument(err.empty() ? "analysis failed" : err);
  auto P = std::make_shared<Plan>();
  P->build(std::move(S), stream_);
  adopt(std::move(P));
  return kOk;
}

void Solver::adopt(std::shared_ptr<Plan> P) {
  MPIR_CUDA(cudaSetDevice(device));
  const int64_t n = P->S.n;
  plan_ = std::move(P);
  // The bfloat16 tier keeps L in bfloat16 for the solves.  The float16 tier
  // does not: float16's range (largest finite 65504) cannot hold the L of
  // these scaled quasi-definite systems, whose entries reach 1/delta-sized
  // values, while bfloat16 has float32's exponent range.
  num_.store_prec = uf == kBF16 ? 2 : 1;
  if (num_.store_prec == 2) {
    // The 16-bit copy sits beside the float32 panels during factorization;
    // where both do not fit, the solves read the float32 panels instead.
    if (Numeric::bytes_for(*plan_, 2) > device_free_bytes(device) / 100 * 97)
      num_.store_prec = 1;
  }
  num_.allocate(*plan_);
  num_.update_mode = update_mode_for(uf, update_engine);
  ws_.allocate(*plan_);
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  vec_.allocate(n, sms);
  vec_m_ = -1;
  // The batch buffers belong to the previous pattern.
  bw_  = 0;
  bm_  = -1;
  mws_ = MultiSolveWorkspace{};
  if (wait_ctl_[0] || wait_ctl_[1])
    MPIR_CUDA(cudaMemcpy(ws_.err.as<int32_t>() + 1, wait_ctl_, sizeof wait_ctl_,
                         cudaMemcpyHostToDevice));
}

size_t Solver::device_bytes() const {
  size_t b = num_.device_bytes();
  for (const DeviceBuffer *d : {&ws_.zbuf, &ws_.part, &ws_.sync, &ws_.ready, &ws_.err, &ws_.xbuf,
                                &mws_.zbuf, &mws_.part, &mws_.sync, &mws_.ready, &mws_.err,
                                &vec_.part, &vec_.count, &vec_.infbits, &vecb_.part, &vecb_.count,
                                &vecb_.infbits, &V_, &bs_, &bp_, &ADp_, &x_, &r_, &t_, &d_, &hd_,
                                &y_, &hb_, &hx_, &bV_, &bbs_, &bbp_, &bx_, &br_, &bt_, &bd_, &bhd_,
                                &by_, &bfac_, &bact_, &bkq_, &bin_, &bout_})
    b += d->bytes();
  return b;
}

size_t Solver::bytes_for(const Plan &P, int64_t gmres_iter, int width, int uf) {
  const int64_t n  = std::max<int64_t>(P.S.n, 1);
  const int64_t m  = std::max<int64_t>(std::min(gmres_iter, n), 1);
  size_t        b  = Numeric::bytes_for(P, uf == kBF16 ? 2 : uf == kF16 ? 3 : 1);
  // single-vector workspace and vectors
  b += (std::max<int64_t>(P.S.z_elems, 1) + std::max<int64_t>(P.spart_elems, 1) +
        static_cast<int64_t>(kReadyCopies) * n + n) * sizeof(double);
  b += (m + 1 + 10) * n * sizeof(double) + 2048 * sizeof(double);
  if (width > 1) {
    b += MultiSolveWorkspace::bytes_for(P, width);
    b += (m + 1 + 8) * n * width * sizeof(double) + 2048 * width * sizeof(double);
  }
  return b;
}

void Solver::ensure_vectors() {
  const int64_t n = plan_->S.n, m = std::max<int64_t>(std::min(gmres_iter, n), 1);
  if (vec_m_ == m) return;
  const size_t vb = std::max<int64_t>(n, 1) * sizeof(double);
  V_.resize(vb * (m + 1));
  bs_.resize(vb);
  bp_.resize(vb);
  ADp_.resize(vb);
  x_.resize(vb);
  r_.resize(vb);
  t_.resize(vb);
  d_.resize(vb);
  hb_.resize(vb);
  hx_.resize(vb);
  hd_.resize(sizeof(double) * 2 * (m + 4));
  y_.resize(sizeof(double) * (m + 1));
  vec_m_ = m;
}

int Solver::factor_device(const double *d_Ax) {
  if (!plan_) throw std::logic_error("factor before analyze");
  MPIR_CUDA(cudaSetDevice(device));
  num_.ensure_scratch(*plan_);
  MPIR_CUDA(cudaEventRecord(ev0_, stream_));
  num_.run_graph(*plan_, d_Ax, eps_of(uf), stream_, own_stream_);
  MPIR_CUDA(cudaEventRecord(ev1_, stream_));
  int32_t zc  = 0;
  bool    bad = false;
  last_npos   = num_.result(stream_, &zc, &bad);
  num_.nonfinite = bad;
  float ms    = 0;
  MPIR_CUDA(cudaEventElapsedTime(&ms, ev0_, ev1_));
  last_factor_ms = ms;
  if (last_npos < 0) {
    num_.valid = false;
    return last_npos == -5 ? -5 : kBadInput;
  }
  return kOk;
}

int Solver::factor(const double *Ax) {
  if (!plan_) throw std::logic_error("factor before analyze");
  MPIR_CUDA(cudaSetDevice(device));
  num_.ensure_scratch(*plan_);
  MPIR_CUDA(cudaMemcpyAsync(num_.Ax.as<void>(), Ax, plan_->S.nnz * sizeof(double),
                            cudaMemcpyHostToDevice, stream_));
  return factor_device(num_.Ax.as<double>());
}

void Solver::set_update_engine(int engine) {
  if (engine != kUpdateDefault && engine != kUpdateTF32x3 && engine != kUpdateBF16x3)
    throw std::invalid_argument("update engine: 0 default, 1 3xTF32, 2 3xBF16");
  update_engine = engine;
  if (plan_) num_.update_mode = update_mode_for(uf, engine);
}

double *Solver::values_device() {
  if (!plan_) throw std::logic_error("no analysed pattern");
  num_.ensure_scratch(*plan_);
  return num_.Ax.as<double>();
}

cudaGraph_t Solver::record_factor(int64_t *launches) {
  if (!plan_) throw std::logic_error("factor before analyze");
  MPIR_CUDA(cudaSetDevice(device));
  num_.ensure_scratch(*plan_);
  num_.release_graph();
  return num_.record(*plan_, num_.Ax.as<double>(), eps_of(uf), own_stream_, launches);
}

int Solver::finish_recorded_factor(double ms) {
  num_.eps_uf    = eps_of(uf);
  bool bad       = false;
  last_npos      = num_.result(stream_, nullptr, &bad);
  num_.nonfinite = bad;
  last_factor_ms = ms;
  num_.valid     = last_npos >= 0;
  if (last_npos < 0) return last_npos == -5 ? -5 : kBadInput;
  return kOk;
}

void Solver::set_wait_controls(int poll_log2, int withhold_item) {
  if (!plan_) throw std::logic_error("no analysed pattern");
  MPIR_CUDA(cudaSetDevice(device));
  wait_ctl_[0] = poll_log2;
  wait_ctl_[1] = withhold_item < 0 ? 0 : withhold_item + 1;
  // Words 1 and 2 of each workspace's SolveCtl (word 0 is the error flag);
  // a several-vector workspace allocated later takes them in ensure_batch.
  MPIR_CUDA(cudaMemcpyAsync(ws_.err.as<int32_t>() + 1, wait_ctl_, sizeof wait_ctl_,
                            cudaMemcpyHostToDevice, stream_));
  if (mws_.nr)
    MPIR_CUDA(cudaMemcpyAsync(mws_.err.as<int32_t>() + 1, wait_ctl_, sizeof wait_ctl_,
                              cudaMemcpyHostToDevice, stream_));
  MPIR_CUDA(cudaStreamSynchronize(stream_));
}

// PrecondGmres, gmres_ir.hpp:636-741.
void Solver::precond_gmres(const double *b, double *res, Report &st) {
  const Plan   &P  = *plan_;
  const int64_t n  = P.S.n;
  cudaStream_t  s  = stream_;
  gmres_iter       = std::min<int64_t>(gmres_iter, n);  // gmres_ir.hpp:643
  const int64_t m  = gmres_iter;
  double       *V  = V_.as<double>();
  double       *hd = hd_.as<double>();
  const int64_t *Kp = P.Kp.as<int64_t>();
  const int32_t *Kj = P.Kj.as<int32_t>();
  const double  *Kv = num_.Kval.as<double>();
  MPIR_CUDA(cudaMemsetAsync(res, 0, n * sizeof(double), s));
  auto read = [&](double *h, int first, int cnt) {
    MPIR_CUDA(cudaMemcpyAsync(h, hd + first, cnt * sizeof(double), cudaMemcpyDeviceToHost, s));
    MPIR_CUDA(cudaStreamSynchronize(s));
  };
  double rho;
  vec_.mgs_pass(const_cast<double *>(b), nullptr, nullptr, nullptr, 1, hd, s);
  read(&rho, 0, 1);
  if (rho < tol) return;
  MPIR_CUDA(cudaMemcpyAsync(V, b, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  ldlt_solve_graph(P, num_, V, ws_, s, own_stream_);
  st.precond_applies++;
  vec_.mgs_pass(V, nullptr, nullptr, nullptr, 1, hd, s);
  read(&rho, 0, 1);
  vec_.scale(V, 1 / rho, V, s);

  std::vector<double> H((m + 1) * std::max<int64_t>(m, 1), 0.0), g(m + 1, 0.0),
      c(std::max<int64_t>(m, 1), 0.0), sn(std::max<int64_t>(m, 1), 0.0),
      col(m + 3, 0.0);
  auto h = [&](int64_t i, int64_t j) -> double & { return H[i * std::max<int64_t>(m, 1) + j]; };
  g[0] = rho;
  int64_t k;
  for (k = 0; k < m && rho > tol; k++) {
    double *vk = V + k * n, *w = V + (k + 1) * n;
    vec_.spmv(Kp, Kj, Kv, vk, w, s);
    st.spmv_count++;
    ldlt_solve_graph(P, num_, w, ws_, s, own_stream_);
    st.precond_applies++;
    double *hn = hd + (m + 2);  // normav
    vec_.mgs_pass(w, nullptr, nullptr, nullptr, 1, hn, s);
    vec_.mgs_pass(w, nullptr, nullptr, V, 0, hd, s);
    for (int64_t j = 0; j <= k; j++)
      vec_.mgs_pass(w, V + j * n, hd + j, j < k ? V + (j + 1) * n : nullptr, j < k ? 0 : 1,
                    hd + j + 1, s);
    // The column's k + 2 entries and normav (at m + 2) in one copy.
    read(col.data(), 0, static_cast<int>(m + 3));
    const double normav = col[m + 2];
    for (int64_t j = 0; j <= k + 1; j++) h(j, k) = col[j];
    const double normav2 = h(k + 1, k);
    if (normav + 0.001 * normav2 == normav) {  // Brown/Hindmarsh, gmres_ir.hpp:683
      st.reorth_count++;
      double *h2 = hd + (m + 4);  // second bank is hd[m+4 .. 2m+8)
      vec_.mgs_pass(w, nullptr, nullptr, V, 0, h2, s);
      for (int64_t j = 0; j <= k; j++)
        vec_.mgs_pass(w, V + j * n, h2 + j, j < k ? V + (j + 1) * n : nullptr, j < k ? 0 : 1,
                      h2 + j + 1, s);
      read(col.data(), static_cast<int>(m + 4), static_cast<int>(k + 2));
      for (int64_t j = 0; j <= k; j++) h(j, k) += col[j];
      h(k + 1, k) = col[k + 1];
    }
    if (h(k + 1, k) != 0) vec_.scale(w, 1 / h(k + 1, k), w, s);
    for (int64_t j = 0; j < k; j++) {  // apply previous rotations
      const double w1 = c[j] * h(j, k) - sn[j] * h(j + 1, k);
      const double w2 = sn[j] * h(j, k) + c[j] * h(j + 1, k);
      h(j, k)         = w1;
      h(j + 1, k)     = w2;
    }
    // Dnrm2 of {h_kk, h_k+1,k}, walked last to first as ops.hpp:243 does.
    double nu;
    {
      double scale = 0.0, ssq = 1.0;
      const double pr[2] = {h(k, k), h(k + 1, k)};
      for (int q = 1; q >= 0; q--)
        if (pr[q] != 0.0) {
          const double a = std::fabs(pr[q]);
          if (scale < a) {
            ssq   = 1.0 + ssq * ((scale / a) * (scale / a));
            scale = a;
          } else {
            ssq = ssq + ((a / scale) * (a / scale));
          }
        }
      nu = scale * std::sqrt(ssq);
    }
    if (nu != 0) {
      c[k]            = h(k, k) / nu;
      sn[k]           = -h(k + 1, k) / nu;
      h(k, k)         = c[k] * h(k, k) - sn[k] * h(k + 1, k);
      h(k + 1, k)     = 0.0;
      const double w1 = c[k] * g[k] - sn[k] * g[k + 1];
      const double w2 = sn[k] * g[k] + c[k] * g[k + 1];
      g[k]            = w1;
      g[k + 1]        = w2;
    }
    rho = std::fabs(g[k + 1]);
  }
  st.gmres_iterations += static_cast<int32_t>(k);
  std::vector<double> y(std::max<int64_t>(k, 1), 0.0);
  for (int64_t i = k; i-- > 0;) {
    y[i] = g[i];
    for (int64_t j = i + 1; j < k; j++) y[i] -= h(i, j) * y[j];
    y[i] /= h(i, i);
  }
  if (k > 0) {
    MPIR_CUDA(cudaMemcpyAsync(y_.as<double>(), y.data(), k * sizeof(double),
                              cudaMemcpyHostToDevice, s));
    vec_.combine(V, n, static_cast<int>(k), y_.as<double>(), res, s);
    MPIR_CUDA(cudaStreamSynchronize(s));  // y lives on the host stack
  }
}

// GmresLDLIR::Solve, gmres_ir.hpp:536-634.
int Solver::solve_device(const double *d_b, double *d_x, Report *rep) {
  if (!plan_) throw std::logic_error("solve before analyze");
  if (!num_.valid) throw std::logic_error("solve before a successful factor");
  MPIR_CUDA(cudaSetDevice(device));
  ensure_vectors();
  Report        st;
  st.factor_prec = applied_prec();
  const Plan   &P = *plan_;
  const int64_t n = P.S.n;
  cudaStream_t  s = stream_;
  MPIR_CUDA(cudaEventRecord(ev0_, s));
  const int64_t *Kp = P.Kp.as<int64_t>();
  const int32_t *Kj = P.Kj.as<int32_t>();
  const double  *Kv = num_.Kval.as<double>();
  double *bs = bs_.as<double>(), *x = x_.as<double>(), *r = r_.as<double>(),
         *t = t_.as<double>(), *d = d_.as<double>();
  const bool dd = ur == kDD;
  if (n == 0) {
    if (rep) *rep = st;
    return kOk;
  }
  vec_.rhs_in(P.perm.as<int64_t>(), num_.AD.as<double>(), d_b, bs, ADp_.as<double>(),
              bp_.as<double>(), s);
  double bs_inf;
  vec_.read_inf(&bs_inf, 3, 1, s);
  const auto t_outer = std::chrono::steady_clock::now();
  auto       ms_since = [](std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0)
        .count();
  };
  precond_gmres(bs, x, st);
  vec_.residual(Kp, Kj, Kv, x, bs, r, dd, 0, s);
  st.spmv_count++;
  double r_inf;
  vec_.read_inf(&r_inf, 0, 1, s);
  IrEvent ev;
  ev.initial_residual = r_inf;
  double r_prev = DBL_MAX, r_norm = r_inf / bs_inf;
  const double eps_w = eps_of(uw);
  for (int64_t iter = 1; iter <= ir_iter; iter++) {
    const double scale = r_inf;
    if (scale == 0.0) {  // exact: nothing left to refine
      st.stop_reason = 3;
      break;
    }
    // a non-finite input, or a factor with a pivot beyond its type's range
    if (!std::isfinite(scale) || num_.nonfinite) {
      st.stop_reason = 4;
      break;
    }
    vec_.scale(r, 1.0 / scale, t, s);
    const auto t_inner = std::chrono::steady_clock::now();
    precond_gmres(t, d, st);
    vec_.ir_update(d, scale, x, s);
    double nrm[2];
    vec_.read_inf(nrm, 1, 2, s);
    const double inner_ms = ms_since(t_inner);
    vec_.residual(Kp, Kj, Kv, x, bs, r, dd, 0, s);
    st.spmv_count++;
    vec_.read_inf(&r_inf, 0, 1, s);
    r_norm           = r_inf / bs_inf;
    st.ir_iterations = static_cast<int32_t>(iter);
    ev.iterations.push_back({iter, r_norm, nrm[0], ms_since(t_outer), inner_ms});
    if (nrm[0] <= nrm[1] * (10 * eps_w)) {
      st.stop_reason = 1;
      break;
    }
    if (std::fabs(r_norm - r_prev) < tol) {
      st.stop_reason = 2;
      break;
    }
    r_prev = r_norm;
  }
  st.residual_norm = r_norm;
  ev.stop_reason      = st.stop_reason;
  ev.total_iterations = st.ir_iterations;
  ev.total_time_ms    = ms_since(t_outer);
  log_.push_back(std::move(ev));
  vec_.sol_out(P.perm.as<int64_t>(), ADp_.as<double>(), x, d_x, s);
  vec_.backward_terms(Kp, Kj, num_.Korig.as<double>(), x, ADp_.as<double>(),
                      bp_.as<double>(), s);
  double be[4];
  vec_.read_inf(be, 4, 4, s);
  const double den  = be[1] * be[2] + be[3];
  st.backward_error = den > 0 ? be[0] / den : be[0];
  MPIR_CUDA(cudaEventRecord(ev1_, s));
  MPIR_CUDA(cudaEventSynchronize(ev1_));
  float ms = 0;
  MPIR_CUDA(cudaEventElapsedTime(&ms, ev0_, ev1_));
  st.solve_ms  = ms;
  st.factor_ms = last_factor_ms;
  // A ready-flag wait of the triangular solves that gave up (sticky word).
  int32_t wait_err = 0;
  MPIR_CUDA(cudaMemcpy(&wait_err, ws_.err.as<void>(), sizeof wait_err, cudaMemcpyDeviceToHost));
  if (wait_err != 0) {
    device_zero(ws_.err.as<void>(), sizeof wait_err);
    st.status = -5;
    if (rep) *rep = st;
    return -5;
  }
  if (rep) *rep = st;
  return kOk;
}

// Plain iterative refinement with the LDL^T factor, as LUIR_QDLDL
// (qdldl-luir/luir.hpp:157-236) with residual, working and solution vectors
// in float64: x0 = solve(b); then r = b - A x, d = solve(r / |r|) |r|,
// x += d, until |d| / |x_old| <= 10 eps(float64) or |d| / |d_prev| >= 1/2,
// at most maxiter steps.  The right-hand side of every solve and its result
// are rounded to the factor's type, as the reference keeps them in FACTPREC.
// Runs on the scaled, permuted system; the norms of the stop test are those
// of the unscaled vectors.
int Solver::luir_device(const double *d_b, double *d_x, int maxiter, Report *rep) {
  if (!plan_) throw std::logic_error("solve before analyze");
  if (!num_.valid) throw std::logic_error("solve before factor");
  MPIR_CUDA(cudaSetDevice(device));
  ensure_vectors();
  Report        st;
  st.factor_prec = applied_prec();
  const Plan   &P = *plan_;
  const int64_t n = P.S.n;
  cudaStream_t  s = stream_;
  MPIR_CUDA(cudaEventRecord(ev0_, s));
  if (n == 0) {
    if (rep) *rep = st;
    return kOk;
  }
  const int64_t *Kp = P.Kp.as<int64_t>();
  const int32_t *Kj = P.Kj.as<int32_t>();
  const double  *Kv = num_.Kval.as<double>();
  double *bs = bs_.as<double>(), *x = x_.as<double>(), *r = r_.as<double>(),
         *ADp = ADp_.as<double>();
  vec_.rhs_in(P.perm.as<int64_t>(), num_.AD.as<double>(), d_b, bs, ADp, bp_.as<double>(), s);
  MPIR_CUDA(cudaMemcpyAsync(x, bs, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  vec_.round_to(uf, x, s);
  ldlt_solve_graph(P, num_, x, ws_, s, own_stream_);
  st.precond_applies++;
  vec_.round_to(uf, x, s);
  const double eps = eps_of(kF64);
  double       d0  = DBL_MAX;
  for (int it = 1; it <= maxiter; it++) {
    vec_.residual(Kp, Kj, Kv, x, bs, r, false, 0, s);
    st.spmv_count++;
    vec_.round_to(uf, r, s);
    double rn;
    vec_.read_inf(&rn, 0, 1, s);
    if (rn == 0.0) {
      st.stop_reason = 3;
      break;
    }
    if (!std::isfinite(rn)) {
      st.stop_reason = 4;
      break;
    }
    vec_.scale(r, 1.0 / rn, r, s);
    vec_.round_to(uf, r, s);
    ldlt_solve_graph(P, num_, r, ws_, s, own_stream_);
    st.precond_applies++;
    vec_.round_to(uf, r, s);
    vec_.ir_update(r, rn, x, s, ADp);
    double nrm[2];
    vec_.read_inf(nrm, 1, 2, s);
    st.ir_iterations = it;
    if (nrm[0] / nrm[1] <= 10 * eps) {
      st.stop_reason = 1;
      break;
    }
    if (nrm[0] / d0 >= 0.5) {
      st.stop_reason = 2;
      break;
    }
    d0 = nrm[0];
  }
  vec_.sol_out(P.perm.as<int64_t>(), ADp, x, d_x, s);
  vec_.backward_terms(Kp, Kj, num_.Korig.as<double>(), x, ADp, bp_.as<double>(), s);
  double be[4];
  vec_.read_inf(be, 4, 4, s);
  const double den   = be[1] * be[2] + be[3];
  st.backward_error  = den > 0 ? be[0] / den : be[0];
  st.residual_norm   = be[3] > 0 ? be[0] / be[3] : be[0];  // |b - A x| / |b|
  MPIR_CUDA(cudaEventRecord(ev1_, s));
  MPIR_CUDA(cudaEventSynchronize(ev1_));
  float ms = 0;
  MPIR_CUDA(cudaEventElapsedTime(&ms, ev0_, ev1_));
  st.solve_ms  = ms;
  st.factor_ms = last_factor_ms;
  int32_t wait_err = 0;
  MPIR_CUDA(cudaMemcpy(&wait_err, ws_.err.as<void>(), sizeof wait_err, cudaMemcpyDeviceToHost));
  if (wait_err != 0) {
    device_zero(ws_.err.as<void>(), sizeof wait_err);
    st.status = -5;
    if (rep) *rep = st;
    return -5;
  }
  if (rep) *rep = st;
  return kOk;
}

int Solver::luir(const double *b, double *x, int maxiter, Report *rep) {
  if (!plan_) throw std::logic_error("solve before analyze");
  MPIR_CUDA(cudaSetDevice(device));
  ensure_vectors();
  const int64_t n = plan_->S.n;
  MPIR_CUDA(cudaMemcpyAsync(hb_.as<void>(), b, n * sizeof(double), cudaMemcpyHostToDevice,
                            stream_));
  const int rc = luir_device(hb_.as<double>(), hx_.as<double>(), maxiter, rep);
  MPIR_CUDA(cudaMemcpyAsync(x, hx_.as<void>(), n * sizeof(double), cudaMemcpyDeviceToHost,
                            stream_));
  MPIR_CUDA(cudaStreamSynchronize(stream_));
  return rc;
}

// The residual step of GmresLDLIR::Solve (gmres_ir.hpp:550-551 and :578-579:
// MatrixMultiply then VectorSubtract, ops.hpp:25-45 and :88-96) in the
// residual type, on its own: the k_spmv residual modes over the unscaled
// values, with b and x gathered into the factor's order and r scattered
// back.
double Solver::residual(const double *b, const double *x, double *r, bool dd) {
  if (!plan_) throw std::logic_error("residual before analyze");
  if (!num_.valid) throw std::logic_error("residual before a successful factor");
  MPIR_CUDA(cudaSetDevice(device));
  ensure_vectors();
  const Plan   &P = *plan_;
  const int64_t n = P.S.n;
  if (n == 0) return 0.0;
  cudaStream_t   s    = stream_;
  const int64_t *perm = P.perm.as<int64_t>();
  const double  *AD   = num_.AD.as<double>();
  MPIR_CUDA(cudaMemcpyAsync(hb_.as<void>(), b, n * sizeof(double), cudaMemcpyHostToDevice, s));
  MPIR_CUDA(cudaMemcpyAsync(hx_.as<void>(), x, n * sizeof(double), cudaMemcpyHostToDevice, s));
  vec_.rhs_in(perm, AD, hx_.as<double>(), t_.as<double>(), nullptr, x_.as<double>(), s);
  vec_.rhs_in(perm, AD, hb_.as<double>(), t_.as<double>(), nullptr, bp_.as<double>(), s);
  vec_.residual(P.Kp.as<int64_t>(), P.Kj.as<int32_t>(), num_.Korig.as<double>(),
                x_.as<double>(), bp_.as<double>(), r_.as<double>(), dd, 0, s);
  double rinf = 0;
  vec_.read_inf(&rinf, 0, 1, s);
  vec_.sol_out(perm, nullptr, r_.as<double>(), hx_.as<double>(), s);
  MPIR_CUDA(cudaMemcpyAsync(r, hx_.as<void>(), n * sizeof(double), cudaMemcpyDeviceToHost, s));
  MPIR_CUDA(cudaStreamSynchronize(s));
  return rinf;
}

// The solver log as JSON, the schema of GmresLDLIR::DumpLog
// (gmres_ir.hpp:305-313, events of gmres_ir.hpp:539-632); clears the events.
std::string Solver::dump_log() {
  static const char *reasons[] = {"max_iterations_reached", "converged_small_update",
                                  "converged_residual_stagnation", "exact_residual",
                                  "non_finite_residual"};
  static const char *details[] = {"", "d_norm <= x_norm * (10*eps)",
                                  "abs(r_norm - r_norm_prev) < tol", "r == 0",
                                  "r or the factor is not finite"};
  auto num = [](double v) {
    if (!std::isfinite(v)) return std::string("null");
    char b[64];
    std::snprintf(b, sizeof b, "%.17g", v);
    return std::string(b);
  };
  std::string j = "{\"events\":[";
  for (size_t e = 0; e < log_.size(); e++) {
    const IrEvent &ev = log_[e];
    const int      rs = ev.stop_reason >= 0 && ev.stop_reason <= 4 ? ev.stop_reason : 0;
    j += e ? "," : "";
    j += "{\"name\":\"gmres_ir\",\"initial_residual\":" + num(ev.initial_residual) +
         ",\"iterations\":[";
    for (size_t i = 0; i < ev.iterations.size(); i++) {
      const IrIter &it = ev.iterations[i];
      j += i ? "," : "";
      j += "{\"iteration\":" + std::to_string(it.iteration) + ",\"residual\":" +
           num(it.residual) + ",\"d_norm\":" + num(it.d_norm) + ",\"timestamp_ms\":" +
           num(it.timestamp_ms) + ",\"inner_time_ms\":" + num(it.inner_time_ms) + "}";
    }
    j += "],\"stop_reason\":\"" + std::string(reasons[rs]) + "\"";
    if (rs != 0) j += ",\"stop_reason_detail\":\"" + std::string(details[rs]) + "\"";
    j += ",\"total_iterations\":" + std::to_string(ev.total_iterations) +
         ",\"total_time_ms\":" + num(ev.total_time_ms) + "}";
  }
  j += "],\"max_outer_iterations\":" + std::to_string(ir_iter) +
       ",\"max_inner_iterations\":" + std::to_string(gmres_iter) +
       ",\"tolerance\":" + num(tol) + "}";
  log_.clear();
  return j;
}

int Solver::solve(const double *b, double *x, Report *rep) {
  if (!plan_) throw std::logic_error("solve before analyze");
  MPIR_CUDA(cudaSetDevice(device));
  ensure_vectors();
  const int64_t n = plan_->S.n;
  MPIR_CUDA(cudaMemcpyAsync(hb_.as<void>(), b, n * sizeof(double), cudaMemcpyHostToDevice,
                            stream_));
  const int rc = solve_device(hb_.as<double>(), hx_.as<double>(), rep);
  MPIR_CUDA(cudaMemcpyAsync(x, hx_.as<void>(), n * sizeof(double), cudaMemcpyDeviceToHost,
                            stream_));
  MPIR_CUDA(cudaStreamSynchronize(stream_));
  return rc;
}

}  // namespace mpir
