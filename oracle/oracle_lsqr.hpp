// oracle_lsqr.hpp -- TEST INFRASTRUCTURE ONLY (the oracle): damped LSQR.
//
// The reference calls Krylov.jl (compat "0.10", Project.toml:31; the exact
// patch version is unpinned because Manifest.toml is not committed) through
// `Krylov.krylov_solve!(ws, J_op, mrhs; λ, itmax, atol, btol)` at
// src/photometry/psf_photometry_simultaneous.jl:1222-1224.  This is a
// restatement of the published LSQR algorithm (Paige & Saunders 1982, ACM
// TOMS 8:43-71, with the damping rotation of their section 4) using the
// stopping rules of Krylov.jl's lsqr with its default tolerances:
//   axtol = btol_default = etol = sqrt(eps), conlim = 1/sqrt(eps),
//   rtol = 0, error-bound window = 5; the caller passes atol and btol.
// The iterates are pinned against scipy.sparse.linalg.lsqr (an independent
// Paige-Saunders implementation) in tests/test_oracle_lsqr.py; the exact
// early-exit iteration of Krylov.jl for a truncated solve is unpinned.
#pragma once

#include <cmath>
#include <functional>
#include <vector>

namespace orc {

// Symmetric Givens rotation (Krylov.jl sym_givens / SOL sym_ortho).
inline void sym_givens(double a, double b, double& c, double& s, double& rho) {
    auto sgn = [](double v) { return v > 0 ? 1.0 : (v < 0 ? -1.0 : 0.0); };
    if (b == 0) {
        c = (a == 0) ? 1.0 : sgn(a);
        s = 0;
        rho = std::fabs(a);
    } else if (a == 0) {
        c = 0;
        s = sgn(b);
        rho = std::fabs(b);
    } else if (std::fabs(b) > std::fabs(a)) {
        double t = a / b;
        s = sgn(b) / std::sqrt(1.0 + t * t);
        c = s * t;
        rho = b / s;
    } else {
        double t = b / a;
        c = sgn(a) / std::sqrt(1.0 + t * t);
        s = c * t;
        rho = a / c;
    }
}

struct LsqrStats {
    int iters = 0;
    int status = 0;  // 0 tired, 1 solved, 2 zero-residual, 3 ill-conditioned, 4 trivial (x = 0)
};

// Solves min ||A x - b||^2 + lambda^2 ||x||^2 from x = 0.
// Av(v, out): out = A v (m);  Atu(u, out): out = A' u (n).
LsqrStats lsqr(int64_t m, int64_t n, const std::function<void(const double*, double*)>& Av,
               const std::function<void(const double*, double*)>& Atu, const double* b, double lambda,
               int itmax, double atol, double btol, double* x);

// The same problem by LSMR (solver = :lsmr): Fong & Saunders 2011 (SIAM J. Sci.
// Comput. 33:2950-2971), the damping rotation of their section 3 and the norm /
// condition estimates of their section 4, with Krylov.jl's lsmr stopping rules
// and default tolerances (axtol = btol_default = sqrt(eps), conlim = 1/sqrt(eps),
// rtol = 0; atol and btol from the caller).  Iterates pinned against
// scipy.sparse.linalg.lsmr in tests/test_oracle_operator.py; Krylov.jl's exact
// early-exit iteration for a truncated solve is unpinned.
LsqrStats lsmr(int64_t m, int64_t n, const std::function<void(const double*, double*)>& Av,
               const std::function<void(const double*, double*)>& Atu, const double* b, double lambda,
               int itmax, double atol, double btol, double* x);

}  // namespace orc
