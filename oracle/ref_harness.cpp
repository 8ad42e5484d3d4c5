// Oracle harness: the reference's own CPU code, compiled from its unmodified
// headers, behind a C ABI that the tests and the CPU-baseline timer load with
// ctypes.  Test infrastructure only; nothing in the product links it.
//
// Built by oracle/Makefile into oracle/_ref/libmpir_ref.so from
//   include/MPIR/qdldl.hpp      QDLDL_etree / QDLDL_factor / QDLDL_solve
//   include/MPIR/ops.hpp        MatrixMultiply, Dnrm2, InfNrm, VectorDot
//   include/MPIR/gmres_ir.hpp   GmresLDLIR<UF,UW,UR>::Compute / Solve
//   include/qdldl-luir/luir.hpp LUIR_QDLDL (plain iterative refinement)
// of the reference tree, with oracle/shim/print standing in for <print> and
// oracle/shim/qd/ for the QD library's headers (not installed).
//
// GmresLDLIR keeps its factor in private members and its shipped Compute
// builds an FGPILU factor (gmres_ir.hpp:365-531).  The harness runs Compute
// for the diagonal scaling (gmres_ir.hpp:347-363), then replaces the factor
// members with the QDLDL LDL^T factor of the scaled matrix:
//   Lp_/Li_/Lx_  = CSR of the strictly lower L  (TriangularSolve forward loop,
//                  gmres_ir.hpp:753-761, reads only col < row)
//   Up_/Ui_/Ux_  = CSC of U = D L^T, strictly upper part (gmres_ir.hpp:765-772)
//   UDinv_       = 1/D
// so that Solve (gmres_ir.hpp:536-634) runs GMRES-IR preconditioned by LDL^T,
// the composition the reference's design document specifies
// (docs/Design/SoftDetailedDes/MIS.tex:505-513).  The private members are
// reached through the standard explicit-instantiation access rule, without
// editing the reference headers.
#include <chrono>
#include <cstdint>
#include <cstring>
#include <memory>
#include <print>
#include <stdfloat>
#include <string>
#include <vector>

#include "MPIR/gmres_ir.hpp"
#include "MPIR/ops.hpp"
#include "MPIR/qdldl.hpp"
#include "qdldl-luir/luir.hpp"

using I = int64_t;

// ---- access to GmresLDLIR's private members --------------------------------
template <class Tag, typename Tag::type M>
struct Rob {
  friend typename Tag::type get(Tag) { return M; }
};

#define MPIR_ROB(TAG, CLS, MEMBER, TYPE)     \
  struct TAG {                               \
    using type = TYPE CLS::*;                \
    friend type get(TAG);                    \
  };                                         \
  template struct Rob<TAG, &CLS::MEMBER>;

using S32 = GmresLDLIR<float, double, double>;
using S64 = GmresLDLIR<double, double, double>;
using VZ  = std::vector<std::size_t>;
using VD  = std::vector<double>;
using VF  = std::vector<float>;

MPIR_ROB(S32_n, S32, n_, std::size_t)
MPIR_ROB(S32_Ax, S32, Ax_, VD)
MPIR_ROB(S32_AD, S32, AD_, VD)
MPIR_ROB(S32_Up, S32, Up_, VZ)
MPIR_ROB(S32_Ui, S32, Ui_, VZ)
MPIR_ROB(S32_Ux, S32, Ux_, VF)
MPIR_ROB(S32_UDinv, S32, UDinv_, VF)
MPIR_ROB(S32_Lp, S32, Lp_, VZ)
MPIR_ROB(S32_Li, S32, Li_, VZ)
MPIR_ROB(S32_Lx, S32, Lx_, VF)

MPIR_ROB(S64_n, S64, n_, std::size_t)
MPIR_ROB(S64_Ax, S64, Ax_, VD)
MPIR_ROB(S64_AD, S64, AD_, VD)
MPIR_ROB(S64_Up, S64, Up_, VZ)
MPIR_ROB(S64_Ui, S64, Ui_, VZ)
MPIR_ROB(S64_Ux, S64, Ux_, VD)
MPIR_ROB(S64_UDinv, S64, UDinv_, VD)
MPIR_ROB(S64_Lp, S64, Lp_, VZ)
MPIR_ROB(S64_Li, S64, Li_, VZ)
MPIR_ROB(S64_Lx, S64, Lx_, VD)

template <class S>
struct Members;
template <>
struct Members<S32> {
  using T = float;
  static auto &Ax(S32 &s) { return s.*get(S32_Ax{}); }
  static auto &AD(S32 &s) { return s.*get(S32_AD{}); }
  static auto &Up(S32 &s) { return s.*get(S32_Up{}); }
  static auto &Ui(S32 &s) { return s.*get(S32_Ui{}); }
  static auto &Ux(S32 &s) { return s.*get(S32_Ux{}); }
  static auto &UDinv(S32 &s) { return s.*get(S32_UDinv{}); }
  static auto &Lp(S32 &s) { return s.*get(S32_Lp{}); }
  static auto &Li(S32 &s) { return s.*get(S32_Li{}); }
  static auto &Lx(S32 &s) { return s.*get(S32_Lx{}); }
};
template <>
struct Members<S64> {
  using T = double;
  static auto &Ax(S64 &s) { return s.*get(S64_Ax{}); }
  static auto &AD(S64 &s) { return s.*get(S64_AD{}); }
  static auto &Up(S64 &s) { return s.*get(S64_Up{}); }
  static auto &Ui(S64 &s) { return s.*get(S64_Ui{}); }
  static auto &Ux(S64 &s) { return s.*get(S64_Ux{}); }
  static auto &UDinv(S64 &s) { return s.*get(S64_UDinv{}); }
  static auto &Lp(S64 &s) { return s.*get(S64_Lp{}); }
  static auto &Li(S64 &s) { return s.*get(S64_Li{}); }
  static auto &Lx(S64 &s) { return s.*get(S64_Lx{}); }
};

static double now_s() {
  using C = std::chrono::steady_clock;
  return std::chrono::duration<double>(C::now().time_since_epoch()).count();
}

// ---- QDLDL ------------------------------------------------------------------
template <class P>
static I factor_as(I n, const I *Ap, const I *Ai, const double *Ax, I *Lp,
                   I *Li, P *Lx, P *D, P *Dinv, const I *Lnz, const I *etree) {
  const I        nnz = Ap[n];
  std::vector<P> a(static_cast<std::size_t>(nnz));
  for (I p = 0; p < nnz; p++) a[p] = static_cast<P>(Ax[p]);
  std::unique_ptr<bool[]> bwork(new bool[n > 0 ? n : 1]);
  std::vector<I>          iwork(3 * static_cast<std::size_t>(n) + 1);
  std::vector<P>          fwork(static_cast<std::size_t>(n) + 1);
  return QDLDL_factor<I, P>(n, Ap, Ai, a.data(), Lp, Li, Lx, D, Dinv, Lnz,
                            etree, bwork.get(), iwork.data(), fwork.data());
}

extern "C" {

I ref_qdldl_etree(I n, const I *Ap, const I *Ai, I *work, I *Lnz, I *etree) {
  return QDLDL_etree<I>(n, Ap, Ai, work, Lnz, etree);
}

I ref_qdldl_factor_f64(I n, const I *Ap, const I *Ai, const double *Ax, I *Lp,
                       I *Li, double *Lx, double *D, double *Dinv,
                       const I *Lnz, const I *etree) {
  return factor_as<double>(n, Ap, Ai, Ax, Lp, Li, Lx, D, Dinv, Lnz, etree);
}

I ref_qdldl_factor_f32(I n, const I *Ap, const I *Ai, const double *Ax, I *Lp,
                       I *Li, float *Lx, float *D, float *Dinv, const I *Lnz,
                       const I *etree) {
  return factor_as<float>(n, Ap, Ai, Ax, Lp, Li, Lx, D, Dinv, Lnz, etree);
}

// 16-bit factors travel as raw bit patterns (uint16_t) through the C ABI.
I ref_qdldl_factor_bf16(I n, const I *Ap, const I *Ai, const double *Ax, I *Lp,
                        I *Li, uint16_t *Lx, uint16_t *D, uint16_t *Dinv,
                        const I *Lnz, const I *etree) {
  static_assert(sizeof(std::bfloat16_t) == 2);
  return factor_as<std::bfloat16_t>(
      n, Ap, Ai, Ax, Lp, Li, reinterpret_cast<std::bfloat16_t *>(Lx),
      reinterpret_cast<std::bfloat16_t *>(D),
      reinterpret_cast<std::bfloat16_t *>(Dinv), Lnz, etree);
}

I ref_qdldl_factor_f16(I n, const I *Ap, const I *Ai, const double *Ax, I *Lp,
                       I *Li, uint16_t *Lx, uint16_t *D, uint16_t *Dinv,
                       const I *Lnz, const I *etree) {
  static_assert(sizeof(std::float16_t) == 2);
  return factor_as<std::float16_t>(
      n, Ap, Ai, Ax, Lp, Li, reinterpret_cast<std::float16_t *>(Lx),
      reinterpret_cast<std::float16_t *>(D),
      reinterpret_cast<std::float16_t *>(Dinv), Lnz, etree);
}

void ref_qdldl_solve_f64_f64(I n, const I *Lp, const I *Li, const double *Lx,
                             const double *Dinv, double *x) {
  QDLDL_solve<I, double, double>(n, Lp, Li, Lx, Dinv, x);
}
void ref_qdldl_solve_f32_f64(I n, const I *Lp, const I *Li, const float *Lx,
                             const float *Dinv, double *x) {
  QDLDL_solve<I, float, double>(n, Lp, Li, Lx, Dinv, x);
}
void ref_qdldl_solve_f32_f32(I n, const I *Lp, const I *Li, const float *Lx,
                             const float *Dinv, float *x) {
  QDLDL_solve<I, float, float>(n, Lp, Li, Lx, Dinv, x);
}
void ref_qdldl_solve_bf16_f32(I n, const I *Lp, const I *Li,
                              const uint16_t *Lx, const uint16_t *Dinv,
                              float *x) {
  QDLDL_solve<I, std::bfloat16_t, float>(
      n, Lp, Li, reinterpret_cast<const std::bfloat16_t *>(Lx),
      reinterpret_cast<const std::bfloat16_t *>(Dinv), x);
}
void ref_qdldl_solve_f16_f32(I n, const I *Lp, const I *Li, const uint16_t *Lx,
                             const uint16_t *Dinv, float *x) {
  QDLDL_solve<I, std::float16_t, float>(
      n, Lp, Li, reinterpret_cast<const std::float16_t *>(Lx),
      reinterpret_cast<const std::float16_t *>(Dinv), x);
}

// Time QDLDL_factor<float> on the leading k x k principal block of an upper
// CSC matrix.  The up-looking factor computes row k of L from rows < k only
// (qdldl.hpp:228-342), so this is exactly the time the full factor spends on
// its first k rows.  Returns seconds, or -1 on a factor error.
double ref_time_factor_leading_f32(I k, const I *Ap, const I *Ai,
                                   const double *Ax) {
  std::vector<I> work(k + 1), Lnz(k + 1), etree(k + 1);
  I sum = QDLDL_etree<I>(k, Ap, Ai, work.data(), Lnz.data(), etree.data());
  if (sum < 0) return -1.0;
  std::vector<I>     Lp(k + 1), Li(sum > 0 ? sum : 1);
  std::vector<float> Lx(sum > 0 ? sum : 1), D(k + 1), Dinv(k + 1);
  const double       t0 = now_s();
  I r = factor_as<float>(k, Ap, Ai, Ax, Lp.data(), Li.data(), Lx.data(),
                         D.data(), Dinv.data(), Lnz.data(), etree.data());
  const double t1 = now_s();
  return r < 0 ? -1.0 : t1 - t0;
}

// ---- ops.hpp ------------------------------------------------------------------
void ref_matmul(I n, const I *Ap, const I *Ai, const double *Ax,
                const double *x, double *y) {
  VZ ap(Ap, Ap + n + 1), ai(Ai, Ai + Ap[n]);
  VD ax(Ax, Ax + Ap[n]), xv(x, x + n);
  VD r = MatrixMultiply<double>(ap, ai, ax, xv);
  std::memcpy(y, r.data(), sizeof(double) * n);
}
double ref_dnrm2(I n, const double *x) {
  return Dnrm2<double>(VD(x, x + n));
}
double ref_infnrm(I n, const double *x) { return InfNrm(VD(x, x + n)); }
double ref_dot(I n, const double *a, const double *b) {
  return VectorDot<double>(VD(a, a + n), VD(b, b + n));
}
float ref_dot_f32(I n, const float *a, const float *b) {
  return VectorDot<float>(VF(a, a + n), VF(b, b + n));
}
double ref_dot_f32_f64(I n, const float *a, const double *b) {
  return VectorDot<double>(VF(a, a + n), VD(b, b + n));
}
// op: 0 add, 1 subtract, 2 multiply (element-wise), 3 scale by b[0]
void ref_vector_op(int op, I n, const double *a, const double *b, double *c) {
  VD av(a, a + n), r;
  if (op == 3) {
    r = VectorScale<double>(av, b[0]);
  } else {
    VD bv(b, b + n);
    if (op == 0) r = VectorAdd<double>(av, bv);
    if (op == 1) r = VectorSubtract<double>(av, bv);
    if (op == 2) r = VectorMultiply<double>(av, bv);
  }
  std::memcpy(c, r.data(), sizeof(double) * n);
}

}  // extern "C"

// ---- GMRES-IR preconditioned by the QDLDL factor -----------------------------
// Optional outputs: the QDLDL factor of the scaled matrix (L_out / D_out:
// nnz(L) and n entries of T, NULL to skip) and info entries 6 and 7 (the
// QDLDL_etree seconds and the seconds of the shipped Compute, which the
// harness runs only for the diagonal scaling) when info_len >= 8.
template <class S>
static int gmres_ir(I n, const I *Ap, const I *Ai, const double *Ax,
                    const double *b, double *x_out, I ir_iter, I gmres_iter,
                    double tol, double *AD_out, double *info,
                    typename Members<S>::T *L_out = nullptr,
                    typename Members<S>::T *D_out = nullptr, int info_len = 6) {
  using M = Members<S>;
  using T = typename M::T;
  S  s;
  VZ ap(Ap, Ap + n + 1), ai(Ai, Ai + Ap[n]);
  VD ax(Ax, Ax + Ap[n]);
  const double tc0 = now_s();
  s.template Compute<double, (std::size_t{1} << 21), 1, 64>(ap, ai, ax, 0);
  const double tc1 = now_s();

  // QDLDL on the scaled matrix the solver holds.
  const VD      &axs = M::Ax(s);
  std::vector<I> work(n), Lnz(n), et(n);
  const double   te0 = now_s();
  I sum = QDLDL_etree<I>(n, Ap, Ai, work.data(), Lnz.data(), et.data());
  const double   te1 = now_s();
  if (sum < 0) return -1;
  std::vector<I> Lp(n + 1), Li(sum > 0 ? sum : 1);
  std::vector<T> Lx(sum > 0 ? sum : 1), D(n), Dinv(n);
  const double   t0 = now_s();
  I pos = factor_as<T>(n, Ap, Ai, axs.data(), Lp.data(), Li.data(), Lx.data(),
                       D.data(), Dinv.data(), Lnz.data(), et.data());
  const double t1 = now_s();
  if (pos < 0) return -2;
  if (L_out && sum > 0) std::memcpy(L_out, Lx.data(), sizeof(T) * sum);
  if (D_out) std::memcpy(D_out, D.data(), sizeof(T) * n);
  if (info && info_len >= 8) {
    info[6] = te1 - te0;
    info[7] = tc1 - tc0;
  }

  // CSR of strictly lower L = transpose of QDLDL's CSC.
  VZ             rp(n + 1, 0), ci(sum > 0 ? sum : 0);
  std::vector<T> rv(sum > 0 ? sum : 0), uv(sum > 0 ? sum : 0);
  for (I p = 0; p < sum; p++) rp[Li[p] + 1]++;
  for (I i = 0; i < n; i++) rp[i + 1] += rp[i];
  VZ fill(rp.begin(), rp.end() - 1);
  for (I j = 0; j < n; j++)
    for (I p = Lp[j]; p < Lp[j + 1]; p++) {
      const std::size_t q = fill[Li[p]]++;
      ci[q]               = static_cast<std::size_t>(j);
      rv[q]               = Lx[p];
      uv[q]               = static_cast<T>(D[j] * Lx[p]);  // U = D L^T
    }
  M::Lp(s)    = rp;
  M::Li(s)    = ci;
  M::Lx(s)    = rv;
  M::Up(s)    = rp;  // column c of U = row c of L, scaled by D of the row
  M::Ui(s)    = ci;
  M::Ux(s)    = uv;
  M::UDinv(s) = Dinv;

  s.SetMaxIRIterations(static_cast<std::size_t>(ir_iter));
  s.SetMaxGmresIterations(static_cast<std::size_t>(gmres_iter));
  s.SetTolerance(tol);
  mpir_shim::capture = true;
  mpir_shim::lines.clear();
  const double t2 = now_s();
  VD           x  = s.Solve(VD(b, b + n));
  const double t3 = now_s();
  mpir_shim::capture = false;
  I ir_steps = 0, reorth = 0;
  for (const auto &l : mpir_shim::lines) {
    if (l.rfind("relative residual", 0) == 0) ir_steps++;
    if (l.rfind("reorth", 0) == 0) reorth++;
  }
  if (x.size() != static_cast<std::size_t>(n)) return -3;
  std::memcpy(x_out, x.data(), sizeof(double) * n);
  if (AD_out) std::memcpy(AD_out, M::AD(s).data(), sizeof(double) * n);
  if (info) {
    info[0] = t1 - t0;  // factor seconds
    info[1] = t3 - t2;  // solve seconds
    info[2] = static_cast<double>(ir_steps);
    info[3] = static_cast<double>(reorth);
    info[4] = static_cast<double>(sum);
    info[5] = static_cast<double>(pos);
  }
  return 0;
}

extern "C" {
// Returns 0 on success; info = {factor_s, solve_s, ir_steps, reorth, nnzL, #D>0}.
int ref_gmres_ir_f32(I n, const I *Ap, const I *Ai, const double *Ax,
                     const double *b, double *x, I ir_iter, I gmres_iter,
                     double tol, double *AD_out, double *info) {
  return gmres_ir<S32>(n, Ap, Ai, Ax, b, x, ir_iter, gmres_iter, tol, AD_out,
                       info);
}
int ref_gmres_ir_f64(I n, const I *Ap, const I *Ai, const double *Ax,
                     const double *b, double *x, I ir_iter, I gmres_iter,
                     double tol, double *AD_out, double *info) {
  return gmres_ir<S64>(n, Ap, Ai, Ax, b, x, ir_iter, gmres_iter, tol, AD_out,
                       info);
}
// As ref_gmres_ir_f32, also returning the float32 factor values of the scaled
// matrix (Lx in QDLDL's CSC order, D) and info[6] = QDLDL_etree seconds,
// info[7] = seconds of the shipped Compute (info holds 8 entries).
int ref_gmres_ir_f32_ex(I n, const I *Ap, const I *Ai, const double *Ax,
                        const double *b, double *x, I ir_iter, I gmres_iter,
                        double tol, double *AD_out, double *info, float *Lx,
                        float *D) {
  return gmres_ir<S32>(n, Ap, Ai, Ax, b, x, ir_iter, gmres_iter, tol, AD_out,
                       info, Lx, D, 8);
}
}  // extern "C"

extern "C" {
// LUIR_QDLDL<float, double, double, double> on A (upper CSC, natural order).
// info = {num_refinement_steps_, relative_residual_, Lnz_}.
int ref_luir_qdldl_f32(I n, const I *Ap, const I *Ai, const double *Ax, const double *b,
                       double *x, int maxiter, double *info) {
  Stats st;
  LUIR_QDLDL<float, double, double, double, I>(n, Ap, Ai, Ax, b, x, &st, maxiter);
  info[0] = st.num_refinement_steps_;
  info[1] = st.relative_residual_;
  info[2] = static_cast<double>(st.Lnz_);
  return 0;
}
}  // extern "C"
