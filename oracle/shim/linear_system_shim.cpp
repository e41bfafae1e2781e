// Replacement for the reference's src/core/LinearSystem.cpp, used only to
// compile the reference's own groundwater sources into the test oracle
// (oracle/_ref).  The class declaration is the reference's own
// (core/LinearSystem.hpp); the PETSc KSP it wraps is not available here, so
// this file restates the PETSc 3.2x algorithms the reference configures:
//
//  * KSPCG, Hestenes-Stiefel form (PETSc src/ksp/ksp/impls/cg/cg.c): zero
//    initial guess, preconditioned residual norm ||B r||, beta = z'r,
//    p = z + (beta/betaold) p, a = beta / p'Ap, the indefinite-matrix and
//    indefinite-PC breakdown checks, DIVERGED_ITS at max_it.
//  * KSPConvergedDefault: converged when ||B r_k|| <= max(rtol ||B b||, atol),
//    diverged when ||B r_k|| >= 1e5 ||B b|| or non-finite.
//  * PCJACOBI: z = r .* (1 / diag(A)), a zero diagonal treated as 1.
//  * PCBJACOBI + ICC(0) on one rank (= global ICC(0), natural ordering) built
//    from the upper triangle of A.  The 7-point graph has no triangles, so
//    IC(0) is d_m = a_mm - sum_{l<m} a_lm^2 / d_l and the apply is the
//    forward/backward substitution with L = I + U^T D^-1.
//  * MatSetValuesCOO with INSERT_VALUES: duplicate (row, col) entries are
//    summed, negative column indices are ignored.
//
// Call sites in the reference: LinearSystem.cpp:147-151 (KSPCG + tolerances),
// :158-226 (PC selection), :294 and :308 (COO), :320 (KSPSolve).
// The preconditioner lane is chosen with frehg_shim_set_pc("jacobi"|"icc")
// (the reference's `-gw_pc_type jacobi` option); the default is the
// reference default bjacobi-icc.

#include "core/Config.hpp"
#include "core/LinearSystem.hpp"
#include "core/Logger.hpp"

#include <chrono>
#include <cmath>
#include <filesystem>
#include <map>
#include <string>
#include <vector>

namespace frehg_shim {
std::string g_pcOverride;  // "" = use settings.preconditioner
}  // namespace frehg_shim

extern "C" void frehg_shim_set_pc(const char* pc) { frehg_shim::g_pcOverride = pc ? pc : ""; }

namespace {

struct Csr {
  int n = 0;
  std::vector<int> rowPtr;
  std::vector<int> col;
  std::vector<double> val;
  std::vector<long long> cooSlot;  // COO entry -> CSR slot (-1 = ignored)
};

struct ShimState {
  Csr a;
  std::vector<double> diagInv;  // Jacobi
  std::vector<double> iccD;     // ICC(0) pivots
  bool jacobi = false;
  double rtol = 1e-8, atol = 1e-14, dtol = 1e5;
  int maxIt = 1000;
  std::vector<double> b, x;
};

std::map<const frehg::LinearSystem*, ShimState>& states() {
  static std::map<const frehg::LinearSystem*, ShimState> s;
  return s;
}

double nowSeconds() {
  using clock = std::chrono::steady_clock;
  return std::chrono::duration<double>(clock::now().time_since_epoch()).count();
}

// The OpenMP build (the CPU-baseline timing lane) runs the vector kernels
// of the solve -- SpMV, dot products, AXPYs, the Jacobi apply -- across the
// host threads, as PETSc's aijkokkos does on a Kokkos-OpenMP host; the ICC(0)
// triangular solves stay serial, as PETSc's are.  The serial build (the
// parity oracle) keeps one fixed summation order.
#ifdef FREHG_SHIM_OPENMP
#define SHIM_PAR_FOR _Pragma("omp parallel for schedule(static)")
#define SHIM_PAR_SUM _Pragma("omp parallel for schedule(static) reduction(+ : s)")
#else
#define SHIM_PAR_FOR
#define SHIM_PAR_SUM
#endif

void spmv(const Csr& a, const double* x, double* y) {
  SHIM_PAR_FOR
  for (int m = 0; m < a.n; ++m) {
    double s = 0.0;
    for (int q = a.rowPtr[m]; q < a.rowPtr[m + 1]; ++q) s += a.val[q] * x[a.col[q]];
    y[m] = s;
  }
}

double dot(const std::vector<double>& u, const std::vector<double>& v) {
  double s = 0.0;
  const long nn = static_cast<long>(u.size());
  SHIM_PAR_SUM
  for (long n = 0; n < nn; ++n) s += u[n] * v[n];
  return s;
}

void applyPc(const ShimState& st, const std::vector<double>& r, std::vector<double>& z) {
  const int n = st.a.n;
  if (st.jacobi) {
    SHIM_PAR_FOR
    for (int m = 0; m < n; ++m) z[m] = r[m] * st.diagInv[m];
    return;
  }
  // L y = r with L = I + U^T D^-1 (lower entries come from the upper triangle).
  std::vector<double> y(r);
  for (int m = 0; m < n; ++m) {
    for (int q = st.a.rowPtr[m]; q < st.a.rowPtr[m + 1]; ++q) {
      const int c = st.a.col[q];
      if (c > m) y[c] -= st.a.val[q] / st.iccD[m] * y[m];
    }
  }
  // L^T z = D^-1 y, backward.
  for (int m = n - 1; m >= 0; --m) {
    double s = y[m] / st.iccD[m];
    for (int q = st.a.rowPtr[m]; q < st.a.rowPtr[m + 1]; ++q) {
      const int c = st.a.col[q];
      if (c > m) s -= st.a.val[q] / st.iccD[m] * z[c];
    }
    z[m] = s;
  }
}

}  // namespace

namespace frehg {

std::string FrehgConfig::resolvePath(const std::string& relative) const {
  if (!relative.empty() && relative[0] == '/') return relative;
  return (std::filesystem::path(configDir) / relative).string();
}

LinearSystem::LinearSystem(MPI_Comm comm, const std::string& prefix, PetscInt nLocalRows,
                           PetscInt nGlobalRows, const SolverSettings& settings)
    : comm_(comm), prefix_(prefix), nLocalRows_(nLocalRows), nGlobalRows_(nGlobalRows) {
  if (nLocalRows_ < 0 || nGlobalRows_ < 1) {
    log::fatal(log::msg() << "LinearSystem('" << prefix_ << "'): invalid sizes");
  }
  ShimState& st = states()[this];
  std::string pc = settings.preconditioner;
  if (!frehg_shim::g_pcOverride.empty()) pc = frehg_shim::g_pcOverride;
  if (pc == "jacobi") {
    st.jacobi = true;
  } else if (pc == "bjacobi-icc" || pc == "icc") {
    st.jacobi = false;
  } else {
    log::fatal(log::msg() << "LinearSystem shim: preconditioner '" << pc
                          << "' is not restated (jacobi | bjacobi-icc)");
  }
  st.rtol = settings.rtol;
  st.atol = settings.atol;
  st.maxIt = settings.maxIterations;
  matType_ = "aij";
  reusable_ = false;
}

LinearSystem::~LinearSystem() { states().erase(this); }

void LinearSystem::setPattern(const Kokkos::View<PetscInt*, MemSpace>& cooRows,
                              const Kokkos::View<PetscInt*, MemSpace>& cooCols) {
  ShimState& st = states()[this];
  const std::size_t nc = cooRows.extent(0);
  const int n = nLocalRows_;
  std::vector<std::map<int, int>> rows(static_cast<std::size_t>(n));
  for (std::size_t e = 0; e < nc; ++e) {
    const int r = cooRows(e), c = cooCols(e);
    if (r < 0 || c < 0) continue;
    rows[static_cast<std::size_t>(r)].emplace(c, 0);
  }
  Csr& a = st.a;
  a.n = n;
  a.rowPtr.assign(static_cast<std::size_t>(n) + 1, 0);
  for (int m = 0; m < n; ++m) {
    int q = a.rowPtr[m];
    for (auto& kv : rows[static_cast<std::size_t>(m)]) {
      kv.second = q++;
      a.col.push_back(kv.first);
    }
    a.rowPtr[m + 1] = q;
  }
  a.val.assign(a.col.size(), 0.0);
  a.cooSlot.assign(nc, -1);
  for (std::size_t e = 0; e < nc; ++e) {
    const int r = cooRows(e), c = cooCols(e);
    if (r < 0 || c < 0) continue;
    a.cooSlot[e] = rows[static_cast<std::size_t>(r)][c];
  }
  nCoo_ = static_cast<PetscCount>(nc);
  patternSet_ = true;
}

void LinearSystem::setValues(const Kokkos::View<real_t*, MemSpace>& values) {
  if (!patternSet_) {
    log::fatal(log::msg() << "LinearSystem('" << prefix_ << "'): setValues before setPattern");
  }
  ShimState& st = states()[this];
  std::fill(st.a.val.begin(), st.a.val.end(), 0.0);
  for (std::size_t e = 0; e < st.a.cooSlot.size(); ++e) {
    if (st.a.cooSlot[e] >= 0) st.a.val[static_cast<std::size_t>(st.a.cooSlot[e])] += values(e);
  }
}

PetscInt LinearSystem::solveOnce(KSPConvergedReason& reason, PetscReal& residual) {
  ShimState& st = states()[this];
  const int n = st.a.n;
  const double setupStart = nowSeconds();
  // PC setup (PCSetUp_Jacobi / ICC(0) numeric factorization).
  st.diagInv.assign(static_cast<std::size_t>(n), 1.0);
  st.iccD.assign(static_cast<std::size_t>(n), 1.0);
  for (int m = 0; m < n; ++m) {
    double d = 0.0;
    for (int q = st.a.rowPtr[m]; q < st.a.rowPtr[m + 1]; ++q) {
      if (st.a.col[q] == m) d = st.a.val[q];
    }
    st.diagInv[m] = (d != 0.0) ? 1.0 / d : 1.0;
    st.iccD[m] = d;
  }
  if (!st.jacobi) {
    for (int m = 0; m < n; ++m) {
      const double dm = st.iccD[m];
      if (!(dm > 0.0)) {
        log::fatal(log::msg() << "ICC(0) shim: non-positive pivot at row " << m);
      }
      for (int q = st.a.rowPtr[m]; q < st.a.rowPtr[m + 1]; ++q) {
        const int c = st.a.col[q];
        if (c > m) st.iccD[c] -= st.a.val[q] * st.a.val[q] / dm;
      }
    }
  }
  telemetry_.setupSeconds += nowSeconds() - setupStart;

  const double solveStart = nowSeconds();
  std::vector<double>& x = st.x;
  const std::vector<double>& b = st.b;
  x.assign(static_cast<std::size_t>(n), 0.0);
  std::vector<double> r(b), z(static_cast<std::size_t>(n)), p(static_cast<std::size_t>(n)),
      w(static_cast<std::size_t>(n));
  applyPc(st, r, z);
  double dp = std::sqrt(dot(z, z));
  reason = KSP_CONVERGED_ITERATING;
  PetscInt its = 0;
  const double rnorm0 = dp;
  const double ttol = std::max(st.rtol * rnorm0, st.atol);
  const auto test = [&](double rn) {
    if (!std::isfinite(rn)) {
      reason = KSP_DIVERGED_NANORINF;
    } else if (rn <= ttol) {
      reason = (rn < st.atol) ? KSP_CONVERGED_ATOL : KSP_CONVERGED_RTOL;
    } else if (rn >= st.dtol * rnorm0) {
      reason = KSP_DIVERGED_DTOL;
    }
  };
  test(dp);
  if (reason == KSP_CONVERGED_ITERATING) {
    double beta = dot(z, r), betaold = 1.0, dpi = 0.0, dpiold = 0.0;
    int i = 0;
    do {
      its = i + 1;
      if (beta == 0.0) {
        reason = KSP_CONVERGED_ATOL;
        break;
      } else if (i > 0 && beta * betaold < 0.0) {
        reason = KSP_DIVERGED_INDEFINITE_PC;
        break;
      }
      if (i == 0) {
        p = z;
      } else {
        const double bb = beta / betaold;
        SHIM_PAR_FOR
        for (int m = 0; m < n; ++m) p[m] = z[m] + bb * p[m];
      }
      dpiold = dpi;
      spmv(st.a, p.data(), w.data());
      dpi = dot(p, w);
      betaold = beta;
      if (dpi == 0.0 || (i > 0 && ((dpi > 0) - (dpi < 0)) * ((dpiold > 0) - (dpiold < 0)) < 0)) {
        reason = KSP_DIVERGED_INDEFINITE_MAT;
        break;
      }
      const double a = beta / dpi;
      SHIM_PAR_FOR
      for (int m = 0; m < n; ++m) x[m] += a * p[m];
      SHIM_PAR_FOR
      for (int m = 0; m < n; ++m) r[m] -= a * w[m];
      applyPc(st, r, z);
      dp = std::sqrt(dot(z, z));
      test(dp);
      if (reason != KSP_CONVERGED_ITERATING) break;
      beta = dot(z, r);
      ++i;
    } while (i < st.maxIt);
    if (i >= st.maxIt) reason = KSP_DIVERGED_ITS;
  }
  residual = dp;
  telemetry_.solveSeconds += nowSeconds() - solveStart;
  return its;
}

SolveStats LinearSystem::solve(const Kokkos::View<real_t*, MemSpace>& rhs,
                               const Kokkos::View<real_t*, MemSpace>& solution) {
  if (rhs.extent(0) != static_cast<std::size_t>(nLocalRows_) ||
      solution.extent(0) != static_cast<std::size_t>(nLocalRows_)) {
    log::fatal(log::msg() << "LinearSystem('" << prefix_ << "'): rhs/solution size mismatch");
  }
  ShimState& st = states()[this];
  st.b.assign(rhs.data(), rhs.data() + nLocalRows_);
  KSPConvergedReason reason = KSP_CONVERGED_ITERATING;
  PetscReal residual = 0.0;
  const PetscInt iterations = solveOnce(reason, residual);
  if (reason < 0) {
    log::fatal(log::msg() << "LinearSystem('" << prefix_ << "'): solver diverged after "
                          << iterations << " iterations, residual " << residual << ", reason "
                          << static_cast<int>(reason));
  }
  ++telemetry_.rebuilds;
  ++telemetry_.solves;
  telemetry_.totalIterations += static_cast<long>(iterations);
  telemetry_.maxIterations = std::max(telemetry_.maxIterations, static_cast<int>(iterations));
  for (PetscInt m = 0; m < nLocalRows_; ++m) solution(m) = st.x[static_cast<std::size_t>(m)];
  SolveStats stats;
  stats.iterations = static_cast<int>(iterations);
  stats.residualNorm = residual;
  stats.reason = (reason == KSP_CONVERGED_RTOL) ? "CONVERGED_RTOL" : "CONVERGED_ATOL";
  return stats;
}

bool LinearSystem::isSymmetric(real_t tolerance) const {
  const ShimState& st = states().at(this);
  double diff = 0.0, norm = 0.0;
  for (int m = 0; m < st.a.n; ++m) {
    double rowAbs = 0.0, rowDiff = 0.0;
    for (int q = st.a.rowPtr[m]; q < st.a.rowPtr[m + 1]; ++q) {
      const int c = st.a.col[q];
      rowAbs += std::fabs(st.a.val[q]);
      double t = 0.0;
      for (int s = st.a.rowPtr[c]; s < st.a.rowPtr[c + 1]; ++s) {
        if (st.a.col[s] == m) t = st.a.val[s];
      }
      rowDiff += std::fabs(st.a.val[q] - t);
    }
    diff = std::max(diff, rowDiff);
    norm = std::max(norm, rowAbs);
  }
  return diff <= tolerance * (1.0 + norm);
}

}  // namespace frehg
