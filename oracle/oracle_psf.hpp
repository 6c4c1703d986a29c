// oracle_psf.hpp -- TEST INFRASTRUCTURE ONLY (the oracle).
//
// CPU FP64 restatement of the PSF arithmetic CrowdPhot.jl evaluates on the
// fitting hot path.  Only tests/, __graft_entry__.smoke() and bench.py's
// cpu_baseline / reference arm may load the oracle library; the product
// library never includes or links this file.
//
// Parity status: pinned by the restated known-answer tests of the reference
// test suite (noiseless truth recovery, dense-Jacobian identities, finite
// difference gradients, the deterministic ImagePSF fixtures) because the
// Julia reference cannot run in this container; see tests/test_oracle_*.py.
#pragma once

#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

#include "../include/crowdphot_b200.h"

namespace orc {

// One ImagePSF node (src/psf/empirical_models.jl:76-85).
struct Node {
    std::vector<double> data;  // column-major ny x nx
    int64_t ny = 0, nx = 0;
    double oy = 0, ox = 0;     // origin.y, origin.x
    double sx = 1, sy = 1;     // oversampling[1] (x), oversampling[2] (y)
    double fill = 0;
    double at(int64_t i, int64_t j) const { return data[(i - 1) + (j - 1) * ny]; }  // 1-based
};

// A supported PSF (GriddedPSFModel{ImagePSF} / ImagePSF / CircularGaussianPSF).
struct Psf {
    int kind = 0;
    std::vector<Node> nodes;
    std::vector<double> ygrid, xgrid;  // sorted unique node positions
    std::vector<int> index_grid;       // ny_g x nx_g column-major, 0-based node index
    double fwhm = 0;
};

// Per-star model parameters (the fields ConstructionBase exposes).
struct StarP {
    double y, x, flux, bkg, fwhm;
};

// Julia's GAUSS_PRE = -4*log(2) (src/psf/parametric_models.jl:18).
inline double gauss_pre() { return -4.0 * std::log(2.0); }

// Builds a Psf from the C-ABI descriptor with the reference's constructor checks
// (gridded_psf.jl:64-135; empirical_models.jl:91-140).  Returns "" on success.
std::string load_psf(const cpb_psf_desc* d, Psf& out);

// _cubic4 (empirical_models.jl:185-196): value and derivative.
inline void cubic4(double f1, double f2, double f3, double f4, double t, double& value, double& deriv) {
    double c1 = (f3 - f1) / 2;
    double c4 = f3 - f2 - c1;
    double c2 = 3 * c4 - (f4 - f2) / 2 + c1;
    double c3 = c4 - c2;
    double c4t = t * c3;
    value = t * (t * (c4t + c2) + c1) + f2;
    deriv = t * (3 * c4t + 2 * c2) + c1;
}

// bicubic_interpolate (empirical_models.jl:239-292).
void bicubic(const double* data, int64_t ny, int64_t nx, double y, double x, double fill,
             double& v, double& dfdy, double& dfdx);

// One corner pass of _gridded_corner_bicubic_pass! (psf_fitting.jl:1233-1321)
// at a single detector pixel: value, d/dv, d/du of node `nd` recentred on (Y, X).
void corner_point(const Node& nd, double Y, double X, double py, double px,
                  double& pv, double& pdv, double& pdu);

// _grid_corners_dw (gridded_psf.jl:176-208).  idx is 0-based; -1 = inactive.
struct Corner { int idx; double w, dwdy, dwdx; };
void grid_corners_dw(const Psf& psf, double Y, double X, Corner c[4]);

// evaluate / evaluate_fg for the three supported kinds.  g = (df/dy, df/dx, df/dflux).
// Gridded uses the corner-pass arithmetic of the specialised fill/render
// methods (psf_photometry_simultaneous.jl:437-543, 605-673); ImagePSF the
// generic evaluate_fg (empirical_models.jl:304-318); Gaussian
// parametric_models.jl:87-115.
double evaluate(const Psf& psf, const StarP& s, double py, double px);
double evaluate_fg(const Psf& psf, const StarP& s, double py, double px, double g[3]);

// spread_model pieces (oracle_spread.cpp): the band-limited exponential-disk
// kernel, the PSF's Gaussian-equivalent FWHM at (Y, X), the kernel of one fit
// (param NaN: the PSF-derived width; false: spread_model off) and the
// zero-border correlation of an h x w column-major stamp.
void exp_disk_kernel(double fwhm, int half, std::vector<double>& K);
double spread_fwhm(const Psf& psf, double Y, double X);
bool spread_kernel(const Psf& psf, double param, double y1, double x1, double fit_rad, std::vector<double>& K,
                   int& half);
void correlate_zero(const double* ms, int h, int w, const std::vector<double>& K, int half, double* g);

}  // namespace orc
