// Several GMRES-IR solves with one factor in lockstep.
//
// Each right-hand side runs exactly the control flow of GmresLDLIR::Solve
// (gmres_ir.hpp:536-634) and PrecondGmres (gmres_ir.hpp:636-741) that
// Solver::solve_device runs for one: its own Arnoldi basis, Hessenberg
// matrix, Givens rotations, stop tests and refinement steps.  The vectors of
// the batch sit side by side (vector k at k*n inside blocks of n*width
// doubles), so every vector kernel takes the whole batch in one launch
// (gridDim.y = vectors, finished ones masked), and every preconditioner
// application is one several-vector triangular solve (solve_multi.cu) that
// reads L once for all of them.  Per vector the arithmetic outside the
// preconditioner is that of the single solve; the several-vector triangular
// solve sums in another order, so results agree with one-at-a-time solves to
// rounding, and each vector stops on its own tests.
#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "solver.hpp"

namespace mpir {

size_t Solver::batch_growth(int width) const {
  if (!plan_ || width <= 1) return 0;
  const int64_t n = std::max<int64_t>(plan_->S.n, 1);
  const int64_t m = std::max<int64_t>(std::min(gmres_iter, n), 1);
  if (bw_ == width && bm_ == m) return 0;
  const size_t want = MultiSolveWorkspace::bytes_for(*plan_, width) +
                      static_cast<size_t>(m + 1 + 8) * n * width * sizeof(double) +
                      2048 * width * sizeof(double);
  size_t have = 0;
  for (const DeviceBuffer *d : {&bV_, &bbs_, &bbp_, &bx_, &br_, &bt_, &bd_, &bhd_, &by_, &bfac_,
                                &bact_, &bkq_, &bin_, &bout_, &bpre_, &mws_.zbuf, &mws_.part,
                                &mws_.sync, &mws_.ready, &mws_.err, &mws_.xbuf, &vecb_.part,
                                &vecb_.count, &vecb_.infbits})
    have += d->bytes();
  return want > have ? want - have : 0;
}

void Solver::ensure_batch(int width) {
  ensure_vectors();
  const int64_t n = plan_->S.n, m = std::max<int64_t>(std::min(gmres_iter, n), 1);
  if (bw_ == width && bm_ == m) return;
  const size_t blk = static_cast<size_t>(std::max<int64_t>(n, 1)) * width * sizeof(double);
  bV_.resize(blk * (m + 1));
  bbs_.resize(blk);
  bbp_.resize(blk);
  bx_.resize(blk);
  br_.resize(blk);
  bt_.resize(blk);
  bd_.resize(blk);
  bin_.resize(blk);
  bout_.resize(blk);
  bhd_.resize(sizeof(double) * 2 * (m + 4) * width);
  by_.resize(sizeof(double) * (m + 1) * width);
  bfac_.resize(sizeof(double) * width);
  bact_.resize(sizeof(int32_t) * width);
  bkq_.resize(sizeof(int32_t) * width);
  // Columns that no vector of a call uses stay zero (the several-vector
  // solve reads all width columns).
  MPIR_CUDA(cudaMemsetAsync(bV_.as<void>(), 0, blk * (m + 1), stream_));
  for (DeviceBuffer *b : {&bbs_, &bbp_, &bx_, &br_, &bt_, &bd_})
    MPIR_CUDA(cudaMemsetAsync(b->as<void>(), 0, blk, stream_));
  if (mws_.nr != width) {
    mws_.allocate(*plan_, width);
    MPIR_CUDA(cudaMemcpy(mws_.err.as<int32_t>() + 1, wait_ctl_, sizeof wait_ctl_,
                         cudaMemcpyHostToDevice));
  }
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  vecb_.allocate(n, sms, width);
  if (hpin_) pinned_free(hpin_, hpin_bytes_);
  hpin_ = nullptr;
  // Pinned staging: kStageSlots slots of (width scale factors, width flags)
  // used in turn without waiting (every inner step synchronises once, and
  // takes fewer uploads than slots), then the counts and the coefficients.
  hpin_bytes_ = sizeof(double) * (kStageSlots * 2 * width + width + (m + 1) * width);
  hpin_       = static_cast<double *>(pinned_alloc(hpin_bytes_));
  stage_next_ = 0;
  bw_ = width;
  bm_ = m;
}

void Solver::multi_apply(double *block) {
  ldlt_solve_multi_graph(*plan_, num_, block, bw_, mws_, stream_, own_stream_);
}

void Solver::precond_device(int nrhs, double *d_X) {
  if (!plan_ || !num_.valid) throw std::logic_error("no valid factor");
  MPIR_CUDA(cudaSetDevice(device));
  const int64_t n = plan_->S.n;
  if (nrhs < 1 || nrhs > kMaxBatch) throw std::invalid_argument("1 <= nrhs <= 16");
  if (nrhs == 1) {
    ldlt_solve(*plan_, num_, d_X, ws_, stream_);
  } else {
    const int width = multi_width(nrhs);
    ensure_batch(width);
    double *blk = bt_.as<double>();
    MPIR_CUDA(cudaMemsetAsync(blk, 0, n * width * sizeof(double), stream_));
    MPIR_CUDA(cudaMemcpyAsync(blk, d_X, n * nrhs * sizeof(double), cudaMemcpyDeviceToDevice,
                              stream_));
    multi_apply(blk);
    MPIR_CUDA(cudaMemcpyAsync(d_X, blk, n * nrhs * sizeof(double), cudaMemcpyDeviceToDevice,
                              stream_));
  }
  MPIR_CUDA(cudaStreamSynchronize(stream_));
  int32_t e0 = 0, e1 = 0;
  MPIR_CUDA(cudaMemcpy(&e0, ws_.err.as<void>(), sizeof e0, cudaMemcpyDeviceToHost));
  if (mws_.nr) MPIR_CUDA(cudaMemcpy(&e1, mws_.err.as<void>(), sizeof e1, cudaMemcpyDeviceToHost));
  if (e0 || e1) {
    device_zero(ws_.err.as<void>(), sizeof(int32_t));
    if (mws_.nr) device_zero(mws_.err.as<void>(), sizeof(int32_t));
    throw WaitTimeout();
  }
}

// PrecondGmres (gmres_ir.hpp:636-741) for the vectors k < nb with
// active[k] != 0: b and res are blocks (vector k at k*n).
void Solver::precond_gmres_batch(int nb, const double *b, double *res, std::vector<Report> &st,
                                 const std::vector<int32_t> &active) {
  const Plan    &P  = *plan_;
  const int64_t  n  = P.S.n;
  cudaStream_t   s  = stream_;
  gmres_iter        = std::min<int64_t>(gmres_iter, n);  // gmres_ir.hpp:643
  const int64_t  m  = gmres_iter;
  const int64_t  mm = std::max<int64_t>(m, 1);
  const int      W  = bw_;
  const int64_t  BS = n * W;       // floats between basis blocks
  const int64_t  HS = 2 * (m + 4);  // per-vector bank of H columns and norms
  double        *V  = bV_.as<double>();
  double        *hd = bhd_.as<double>();
  const int64_t *Kp = P.Kp.as<int64_t>();
  const int32_t *Kj = P.Kj.as<int32_t>();
  const double  *Kv = num_.Kval.as<double>();
  int32_t       *hkq  = reinterpret_cast<int32_t *>(hpin_ + kStageSlots * 2 * W);
  double        *hy   = hpin_ + kStageSlots * 2 * W + W;  // width x (m + 1)
  double        *dfac = bfac_.as<double>();
  int32_t       *dact = bact_.as<int32_t>();
  std::vector<double> banks(static_cast<size_t>(HS) * nb);
  auto put_act = [&](const std::vector<int32_t> &a) {
    int32_t *hact = reinterpret_cast<int32_t *>(stage_slot());
    for (int k = 0; k < W; k++) hact[k] = k < nb ? a[k] : 0;
    MPIR_CUDA(cudaMemcpyAsync(dact, hact, W * sizeof(int32_t), cudaMemcpyHostToDevice, s));
  };
  auto put_fac = [&](const std::vector<double> &f) {
    double *hfac = stage_slot();
    for (int k = 0; k < W; k++) hfac[k] = k < nb ? f[k] : 1.0;
    MPIR_CUDA(cudaMemcpyAsync(dfac, hfac, W * sizeof(double), cudaMemcpyHostToDevice, s));
  };
  auto read_banks = [&]() {
    MPIR_CUDA(cudaMemcpyAsync(banks.data(), hd, banks.size() * sizeof(double),
                              cudaMemcpyDeviceToHost, s));
    MPIR_CUDA(cudaStreamSynchronize(s));
  };
  auto bank = [&](int k, int64_t i) -> double { return banks[k * HS + i]; };
  std::vector<int32_t> act = active;
  put_act(act);
  for (int k = 0; k < nb; k++)
    if (act[k]) MPIR_CUDA(cudaMemsetAsync(res + k * n, 0, n * sizeof(double), s));
  std::vector<double> rho(nb, 0.0), fac(nb, 1.0);
  vecb_.mgs_pass_b(nb, const_cast<double *>(b), nullptr, nullptr, nullptr, 1, hd, n, HS, dact, s);
  read_banks();
  for (int k = 0; k < nb; k++)
    if (act[k]) {
      rho[k] = bank(k, 0);
      if (rho[k] < tol) act[k] = 0;  // zero update for this vector
    }
  bool any = false;
  for (int k = 0; k < nb; k++) any |= act[k] != 0;
  if (!any) return;
  put_act(act);
  put_fac(std::vector<double>(nb, 1.0));
  vecb_.scale_b(nb, b, dfac, V, n, dact, s);  // V_0 = b (times 1: bitwise a copy)
  multi_apply(V);
  for (int k = 0; k < nb; k++)
    if (act[k]) st[k].precond_applies++;
  vecb_.mgs_pass_b(nb, V, nullptr, nullptr, nullptr, 1, hd, n, HS, dact, s);
  read_banks();
  for (int k = 0; k < nb; k++)
    if (act[k]) {
      rho[k] = bank(k, 0);
      fac[k] = 1 / rho[k];
    }
  put_fac(fac);
  vecb_.scale_b(nb, V, dfac, V, n, dact, s);

  // Per-vector Hessenberg matrix, rotations and right-hand side (host).
  const int64_t       ld = mm;
  std::vector<std::vector<double>> H(nb, std::vector<double>((m + 1) * ld, 0.0)),
      g(nb, std::vector<double>(m + 1, 0.0)), c(nb, std::vector<double>(mm, 0.0)),
      sn(nb, std::vector<double>(mm, 0.0));
  std::vector<int64_t> kk(nb, 0);
  for (int k = 0; k < nb; k++) g[k][0] = rho[k];
  std::vector<int32_t> inner(nb, 0);
  for (int k = 0; k < nb; k++) inner[k] = act[k] && m > 0 && rho[k] > tol;
  for (int64_t step = 0;; step++) {
    bool more = false;
    for (int k = 0; k < nb; k++) more |= inner[k] != 0;
    if (!more) break;
    put_act(inner);
    double *vk = V + step * BS, *w = V + (step + 1) * BS;
    vecb_.spmv_b(nb, Kp, Kj, Kv, vk, w, n, dact, s);
    multi_apply(w);
    for (int k = 0; k < nb; k++)
      if (inner[k]) {
        st[k].spmv_count++;
        st[k].precond_applies++;
      }
    vecb_.mgs_pass_b(nb, w, nullptr, nullptr, nullptr, 1, hd + (m + 2), n, HS, dact, s);
    vecb_.mgs_pass_b(nb, w, nullptr, nullptr, V, 0, hd, n, HS, dact, s);
    for (int64_t j = 0; j <= step; j++)
      vecb_.mgs_pass_b(nb, w, V + j * BS, hd + j, j < step ? V + (j + 1) * BS : nullptr,
                       j < step ? 0 : 1, hd + j + 1, n, HS, dact, s);
    read_banks();
    std::vector<int32_t> reo(nb, 0);
    bool                 any_reo = false;
    for (int k = 0; k < nb; k++) {
      if (!inner[k]) continue;
      auto         h      = [&](int64_t i, int64_t j) -> double & { return H[k][i * ld + j]; };
      for (int64_t j = 0; j <= step + 1; j++) h(j, step) = bank(k, j);
      const double normav = bank(k, m + 2), normav2 = h(step + 1, step);
      if (normav + 0.001 * normav2 == normav) {  // Brown/Hindmarsh, gmres_ir.hpp:683
        reo[k]  = 1;
        any_reo = true;
      }
    }
    if (any_reo) {
      put_act(reo);
      double *h2 = hd + (m + 4);
      vecb_.mgs_pass_b(nb, w, nullptr, nullptr, V, 0, h2, n, HS, dact, s);
      for (int64_t j = 0; j <= step; j++)
        vecb_.mgs_pass_b(nb, w, V + j * BS, h2 + j, j < step ? V + (j + 1) * BS : nullptr,
                         j < step ? 0 : 1, h2 + j + 1, n, HS, dact, s);
      read_banks();
      for (int k = 0; k < nb; k++) {
        if (!reo[k]) continue;
        st[k].reorth_count++;
        auto h = [&](int64_t i, int64_t j) -> double & { return H[k][i * ld + j]; };
        for (int64_t j = 0; j <= step; j++) h(j, step) += bank(k, m + 4 + j);
        h(step + 1, step) = bank(k, m + 4 + step + 1);
      }
      put_act(inner);
    }
    for (int k = 0; k < nb; k++) {
      if (!inner[k]) continue;
      const double hk = H[k][(step + 1) * ld + step];
      fac[k]          = hk != 0 ? 1 / hk : 1.0;  // times 1: the single solve's skip
    }
    put_fac(fac);
    vecb_.scale_b(nb, w, dfac, w, n, dact, s);
    for (int k = 0; k < nb; k++) {
      if (!inner[k]) continue;
      auto h = [&](int64_t i, int64_t j) -> double & { return H[k][i * ld + j]; };
      for (int64_t j = 0; j < step; j++) {  // apply previous rotations
        const double w1 = c[k][j] * h(j, step) - sn[k][j] * h(j + 1, step);
        const double w2 = sn[k][j] * h(j, step) + c[k][j] * h(j + 1, step);
        h(j, step)      = w1;
        h(j + 1, step)  = w2;
      }
      // Dnrm2 of {h_kk, h_k+1,k}, walked last to first as ops.hpp:243 does.
      double nu;
      {
        double       scale = 0.0, ssq = 1.0;
        const double pr[2] = {h(step, step), h(step + 1, step)};
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
        c[k][step]         = h(step, step) / nu;
        sn[k][step]        = -h(step + 1, step) / nu;
        h(step, step)      = c[k][step] * h(step, step) - sn[k][step] * h(step + 1, step);
        h(step + 1, step)  = 0.0;
        const double w1    = c[k][step] * g[k][step] - sn[k][step] * g[k][step + 1];
        const double w2    = sn[k][step] * g[k][step] + c[k][step] * g[k][step + 1];
        g[k][step]         = w1;
        g[k][step + 1]     = w2;
      }
      rho[k] = std::fabs(g[k][step + 1]);
      kk[k]  = step + 1;
      if (!(kk[k] < m && rho[k] > tol)) inner[k] = 0;
    }
  }
  // Back-substitution and res = V y per vector.
  bool any_y = false;
  MPIR_CUDA(cudaStreamSynchronize(s));
  for (int k = 0; k < W; k++) hkq[k] = 0;
  for (int k = 0; k < nb; k++) {
    if (!act[k]) continue;
    st[k].gmres_iterations += static_cast<int32_t>(kk[k]);
    const int64_t K = kk[k];
    for (int64_t i = K; i-- > 0;) {
      double yi = g[k][i];
      for (int64_t j = i + 1; j < K; j++) yi -= H[k][i * ld + j] * hy[k * (m + 1) + j];
      hy[k * (m + 1) + i] = yi / H[k][i * ld + i];
    }
    hkq[k] = static_cast<int32_t>(K);
    any_y |= K > 0;
  }
  if (any_y) {
    int32_t *hact = reinterpret_cast<int32_t *>(stage_slot());
    for (int k = 0; k < W; k++) hact[k] = k < nb && act[k] && hkq[k] > 0;
    MPIR_CUDA(cudaMemcpyAsync(dact, hact, W * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    MPIR_CUDA(cudaMemcpyAsync(bkq_.as<int32_t>(), hkq, W * sizeof(int32_t),
                              cudaMemcpyHostToDevice, s));
    MPIR_CUDA(cudaMemcpyAsync(by_.as<double>(), hy, W * (m + 1) * sizeof(double),
                              cudaMemcpyHostToDevice, s));
    vecb_.combine_b(nb, V, BS, by_.as<double>(), m + 1, bkq_.as<int32_t>(), res, n, dact, s);
    MPIR_CUDA(cudaStreamSynchronize(s));  // the staging area is reused next
  }
}

// GmresLDLIR::Solve (gmres_ir.hpp:536-634) for nrhs right-hand sides.
int Solver::solve_batch_device(int nrhs, const double *d_B, double *d_X, Report *reps) {
  if (!plan_) throw std::logic_error("solve before analyze");
  if (!num_.valid) throw std::logic_error("solve before a successful factor");
  if (nrhs < 1 || nrhs > kMaxBatch) throw std::invalid_argument("1 <= nrhs <= 16");
  MPIR_CUDA(cudaSetDevice(device));
  const int64_t n = plan_->S.n;
  if (n == 0) {
    for (int k = 0; k < nrhs && reps; k++) reps[k] = Report{};
    return kOk;
  }
  const int W = multi_width(nrhs);
  ensure_batch(W);
  const int    nb = nrhs;
  const Plan  &P  = *plan_;
  cudaStream_t s  = stream_;
  MPIR_CUDA(cudaEventRecord(ev0_, s));
  const int64_t *Kp = P.Kp.as<int64_t>();
  const int32_t *Kj = P.Kj.as<int32_t>();
  const double  *Kv = num_.Kval.as<double>();
  double *bs = bbs_.as<double>(), *x = bx_.as<double>(), *r = br_.as<double>(),
         *t = bt_.as<double>(), *d = bd_.as<double>();
  double *ADp = ADp_.as<double>();
  const bool dd = ur == kDD;
  std::vector<Report> st(nb);
  for (Report &r : st) r.factor_prec = applied_prec();
  std::vector<double> inf(8 * static_cast<size_t>(nb));
  vecb_.rhs_in_b(nb, P.perm.as<int64_t>(), num_.AD.as<double>(), d_B, bs, ADp, bbp_.as<double>(),
                 n, s);
  vecb_.read_inf_b(nb, inf.data(), s);
  std::vector<double> bs_inf(nb);
  for (int k = 0; k < nb; k++) bs_inf[k] = inf[8 * k + 3];
  const auto t_outer  = std::chrono::steady_clock::now();
  auto       ms_since = [](std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0)
        .count();
  };
  std::vector<int32_t> act(nb, 1);
  precond_gmres_batch(nb, bs, x, st, act);
  vecb_.residual_b(nb, Kp, Kj, Kv, x, bs, r, dd, n, nullptr, s);
  vecb_.read_inf_b(nb, inf.data(), s);
  std::vector<double> r_inf(nb), r_prev(nb, DBL_MAX), r_norm(nb);
  std::vector<IrEvent> evs(nb);
  for (int k = 0; k < nb; k++) {
    st[k].spmv_count++;
    r_inf[k]                = inf[8 * k];
    r_norm[k]               = r_inf[k] / bs_inf[k];
    evs[k].initial_residual = r_inf[k];
  }
  const double eps_w = eps_of(uw);
  std::vector<double> fac(nb, 1.0);
  auto put = [&](const std::vector<int32_t> &a, const std::vector<double> &f) {
    double  *hf = stage_slot();
    int32_t *ha = reinterpret_cast<int32_t *>(hf + bw_);
    for (int k = 0; k < bw_; k++) {
      ha[k] = k < nb ? a[k] : 0;
      hf[k] = k < nb ? f[k] : 1.0;
    }
    MPIR_CUDA(cudaMemcpyAsync(bact_.as<void>(), ha, bw_ * sizeof(int32_t),
                              cudaMemcpyHostToDevice, s));
    MPIR_CUDA(cudaMemcpyAsync(bfac_.as<void>(), hf, bw_ * sizeof(double),
                              cudaMemcpyHostToDevice, s));
  };
  for (int64_t iter = 1; iter <= ir_iter; iter++) {
    bool any = false;
    for (int k = 0; k < nb; k++) {
      if (!act[k]) continue;
      const double scale = r_inf[k];
      if (scale == 0.0) {  // exact: nothing left to refine
        st[k].stop_reason = 3;
        act[k]            = 0;
      } else if (!std::isfinite(scale) || num_.nonfinite) {
        st[k].stop_reason = 4;
        act[k]            = 0;
      } else {
        fac[k] = 1.0 / scale;
        any    = true;
      }
    }
    if (!any) break;
    put(act, fac);
    vecb_.scale_b(nb, r, bfac_.as<double>(), t, n, bact_.as<int32_t>(), s);
    const auto t_inner = std::chrono::steady_clock::now();
    precond_gmres_batch(nb, t, d, st, act);
    for (int k = 0; k < nb; k++) fac[k] = r_inf[k];
    put(act, fac);
    vecb_.ir_update_b(nb, d, bfac_.as<double>(), x, n, bact_.as<int32_t>(), s);
    vecb_.read_inf_b(nb, inf.data(), s);
    const double inner_ms = ms_since(t_inner);
    std::vector<double> nrm0(nb), nrm1(nb);
    for (int k = 0; k < nb; k++) {
      nrm0[k] = inf[8 * k + 1];
      nrm1[k] = inf[8 * k + 2];
    }
    vecb_.residual_b(nb, Kp, Kj, Kv, x, bs, r, dd, n, bact_.as<int32_t>(), s);
    vecb_.read_inf_b(nb, inf.data(), s);
    for (int k = 0; k < nb; k++) {
      if (!act[k]) continue;
      st[k].spmv_count++;
      r_inf[k]            = inf[8 * k];
      r_norm[k]           = r_inf[k] / bs_inf[k];
      st[k].ir_iterations = static_cast<int32_t>(iter);
      evs[k].iterations.push_back({iter, r_norm[k], nrm0[k], ms_since(t_outer), inner_ms});
      if (nrm0[k] <= nrm1[k] * (10 * eps_w)) {
        st[k].stop_reason = 1;
        act[k]            = 0;
      } else if (std::fabs(r_norm[k] - r_prev[k]) < tol) {
        st[k].stop_reason = 2;
        act[k]            = 0;
      } else {
        r_prev[k] = r_norm[k];
      }
    }
  }
  vecb_.sol_out_b(nb, P.perm.as<int64_t>(), ADp, x, d_X, n, s);
  vecb_.backward_terms_b(nb, Kp, Kj, num_.Korig.as<double>(), x, ADp, bbp_.as<double>(), n, s);
  vecb_.read_inf_b(nb, inf.data(), s);
  MPIR_CUDA(cudaEventRecord(ev1_, s));
  MPIR_CUDA(cudaEventSynchronize(ev1_));
  float ms = 0;
  MPIR_CUDA(cudaEventElapsedTime(&ms, ev0_, ev1_));
  for (int k = 0; k < nb; k++) {
    const double *be  = inf.data() + 8 * k + 4;
    const double  den = be[1] * be[2] + be[3];
    st[k].backward_error = den > 0 ? be[0] / den : be[0];
    st[k].residual_norm  = r_norm[k];
    st[k].solve_ms       = ms;
    st[k].factor_ms      = last_factor_ms;
    evs[k].stop_reason      = st[k].stop_reason;
    evs[k].total_iterations = st[k].ir_iterations;
    evs[k].total_time_ms    = ms_since(t_outer);
    log_.push_back(std::move(evs[k]));
  }
  int32_t wait_err = 0;
  MPIR_CUDA(cudaMemcpy(&wait_err, mws_.err.as<void>(), sizeof wait_err, cudaMemcpyDeviceToHost));
  const int rc = wait_err != 0 ? -5 : kOk;
  if (wait_err != 0) device_zero(mws_.err.as<void>(), sizeof wait_err);
  for (int k = 0; k < nb; k++) {
    if (rc != kOk) st[k].status = rc;
    if (reps) reps[k] = st[k];
  }
  return rc;
}

int Solver::solve_batch(int nrhs, const double *B, double *X, Report *reps) {
  if (!plan_) throw std::logic_error("solve before analyze");
  if (nrhs < 1 || nrhs > kMaxBatch) throw std::invalid_argument("1 <= nrhs <= 16");
  MPIR_CUDA(cudaSetDevice(device));
  const int64_t n = plan_->S.n;
  ensure_batch(multi_width(nrhs));
  MPIR_CUDA(cudaMemcpyAsync(bin_.as<void>(), B, n * nrhs * sizeof(double), cudaMemcpyHostToDevice,
                            stream_));
  const int rc = solve_batch_device(nrhs, bin_.as<double>(), bout_.as<double>(), reps);
  MPIR_CUDA(cudaMemcpyAsync(X, bout_.as<void>(), n * nrhs * sizeof(double),
                            cudaMemcpyDeviceToHost, stream_));
  MPIR_CUDA(cudaStreamSynchronize(stream_));
  return rc;
}

}  // namespace mpir
