// dmft_loop.cpp — the DMFT self-consistency loop around the impurity solver,
// on the Bethe lattice, in C++ above the library's own C ABI.
//
// Restates the reference's host loop (src/dmft.f90:38-137) for the
// semicircular density of states of half-bandwidth 1 (TBHamiltonian 2,
// src/dmft_lattice.f90:75-103):
//
//   iteration 1:   the initial bath (em, ek, vmk)
//   iteration > 1: fit (em, ek, vmk) to the previous iteration's G_0^-1
//                  corrected by G_loc^-1 - G_cl^-1 (src/ed_projection.f90:23-553),
//                  optionally mixed linearly with the previous parameters
//                  after aligning the fitted bath sites' signs with the
//                  previous ones (mixing 1 reproduces the reference, which
//                  has no mixing)
//   then           D_cl  = sum_l V_l^2 / (i w - e_l)             (dmft_green.f90:24-45)
//                  G_cl  = edzt_ground_state + edzt_cluster_green_ftn
//                  G_loc = int dos(x) / (em + D_cl + 1/G_cl - x) dx  (dmft_green.f90:128-170)
//                  h_imp.dat, green.dat.<o>.<s>, g_coeffs.dat     (dump_data.f90, dmft_green.f90:66-109)
//                  stop when sum |G_cl - G_loc|^2 / (norb nbath nw) < scf_tol   (dmft.f90:105-134)
//   after the loop Sigma = i w + mu - em - D_cl - 1/G_cl, Z = 1/(1 - Im Sigma(i w_1)/w_1),
//                  sigma.dat.<o>.<s>                              (post_process.f90:39-57, :121-185)
//
// The bath fit minimises the reference's cost (src/ed_projection.f90:154-250)
// by a nonlinear conjugate gradient with Polak-Ribiere directions, as the
// reference does, with a line search of this file's own design that uses the
// cost's analytic gradient (fourfold step growth to a bracket, then
// safeguarded Hermite-cubic steps) and the reference's relative stopping
// tolerance (ftol 1e-6 by default).
//
// Array layouts are the reference's Fortran ones: em(norb,2), ek(nbath,2),
// vmk(norb,nbath,2) column-major; complex functions (nw, norb, nspin)
// column-major with interleaved real and imaginary parts.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <string>
#include <vector>
#include "../../include/edzt.h"

// The context's error message (edzt_last_error), set by the library's host code.
void edzt_ctx_set_error(edzt_ctx* c, const char* msg);

namespace {

using cplx = std::complex<double>;

struct Fail {
    int code;
    const char* msg;   // nullptr: the solver call already set the context's message
};

size_t gidx(int iw, int a, int s, int nw, int norb) { return (size_t)iw + (size_t)nw * ((size_t)a + (size_t)norb * s); }

void hybridization(int norb, int nbath, int nspin, int nw, const double* omega, const double* ek, const double* vmk,
                   cplx* D)
{
    for (int s = 0; s < nspin; s++)
        for (int a = 0; a < norb; a++)
            for (int w = 0; w < nw; w++) {
                cplx d = 0.0;
                const cplx iw(0.0, omega[w]);
                for (int l = 0; l < nbath; l++) {
                    const double v = vmk[a + norb * (l + nbath * s)];
                    d += v * v / (iw - ek[l + nbath * s]);
                }
                D[gidx(w, a, s, nw, norb)] = d;
            }
}

// The reference's quadrature: ne equally spaced points on [-1, 1], weights
// 2/pi sqrt(1 - x^2), the sum times 2/(ne - 1).
void local_green(int norb, int nspin, int nw, const double* em, double hfield, const cplx* D, const cplx* Gcl,
                 cplx* Gloc, int ne = 10000)
{
    std::vector<double> x(ne), wt(ne);
    for (int i = 0; i < ne; i++) {
        x[i] = -1.0 + i * 2.0 / (ne - 1);
        wt[i] = 2.0 / M_PI * std::sqrt(std::max(1.0 - x[i] * x[i], 0.0));
    }
    for (int s = 0; s < nspin; s++) {
        const double hs = (s == 0) ? hfield : -hfield;
        for (int a = 0; a < norb; a++)
            for (int w = 0; w < nw; w++) {
                const size_t g = gidx(w, a, s, nw, norb);
                const cplx zeta = em[a + norb * s] + hs + D[g] + 1.0 / Gcl[g];
                cplx sum = 0.0;
                for (int i = 0; i < ne; i++) sum += wt[i] / (zeta - x[i]);
                Gloc[g] = sum * 2.0 / double(ne - 1);
            }
    }
}

double scf_diff(int norb, int nbath, int nspin, int nw, const cplx* Gcl, const cplx* Gloc)
{
    double d = 0.0;
    for (size_t g = 0; g < (size_t)nw * norb * nspin; g++) d += std::norm(Gcl[g] - Gloc[g]);
    return d / ((double)norb * nbath * nw);
}

// Cost and gradient of the fit of spin s (ed_projection.f90:154-250):
// f(x) = sum_{a,w} |em_a - em_old_a + D_a(x) - D_old + 1/G_loc - 1/G_cl|^2 / w
// / (norb nw), x = (em(1..norb), ek(1..nbath), vmk(iorb fastest, ibath)).
struct BathFit {
    int norb, nbath, nw;
    std::vector<double> omega, wgt;
    std::vector<cplx> c;   // [a][w]: -em_old - D_old + 1/G_loc - 1/G_cl

    BathFit(int norb_, int nbath_, int nw_, const double* om, const double* em_old, const cplx* D, const cplx* Gcl,
            const cplx* Gloc, int s)
        : norb(norb_), nbath(nbath_), nw(nw_), omega(om, om + nw_), wgt(nw_), c((size_t)norb_ * nw_)
    {
        for (int w = 0; w < nw; w++) wgt[w] = 1.0 / omega[w];
        for (int a = 0; a < norb; a++)
            for (int w = 0; w < nw; w++) {
                const size_t g = gidx(w, a, s, nw, norb);
                c[(size_t)a * nw + w] = -em_old[a + norb * s] - D[g] + 1.0 / Gloc[g] - 1.0 / Gcl[g];
            }
    }
    double V(const std::vector<double>& x, int a, int l) const { return x[norb + nbath + l * norb + a]; }

    // d[a][w] and den[l][w] = i w - e_l
    void diff(const std::vector<double>& x, std::vector<cplx>& d, std::vector<cplx>& den) const
    {
        den.assign((size_t)nbath * nw, 0.0);
        for (int l = 0; l < nbath; l++)
            for (int w = 0; w < nw; w++) den[(size_t)l * nw + w] = cplx(-x[norb + l], omega[w]);
        d.assign((size_t)norb * nw, 0.0);
        for (int a = 0; a < norb; a++)
            for (int w = 0; w < nw; w++) {
                cplx Dw = 0.0;
                for (int l = 0; l < nbath; l++) {
                    const double v = V(x, a, l);
                    Dw += v * v / den[(size_t)l * nw + w];
                }
                d[(size_t)a * nw + w] = x[a] + Dw + c[(size_t)a * nw + w];
            }
    }
    double f(const std::vector<double>& x) const
    {
        std::vector<cplx> d, den;
        diff(x, d, den);
        double s = 0.0;
        for (int a = 0; a < norb; a++)
            for (int w = 0; w < nw; w++) s += std::norm(d[(size_t)a * nw + w]) * wgt[w];
        return s / ((double)norb * nw);
    }
    std::vector<double> df(const std::vector<double>& x) const
    {
        std::vector<cplx> d, den;
        diff(x, d, den);
        std::vector<double> g(x.size(), 0.0);
        const double scale = 1.0 / ((double)norb * nw);
        for (int a = 0; a < norb; a++) {
            double t = 0.0;
            for (int w = 0; w < nw; w++) t += 2.0 * d[(size_t)a * nw + w].real() * wgt[w];
            g[a] = t * scale;
        }
        for (int l = 0; l < nbath; l++) {
            double te = 0.0;
            for (int a = 0; a < norb; a++) {
                const double v = V(x, a, l);
                double tv = 0.0;
                for (int w = 0; w < nw; w++) {
                    const cplx cden = std::conj(den[(size_t)l * nw + w]);          // -i w - e_l
                    const cplx dw = d[(size_t)a * nw + w];
                    te += 2.0 * (dw * (v * v / (cden * cden))).real() * wgt[w];  // dD/de_l, conjugated
                    tv += 2.0 * (dw * (2.0 * v / cden)).real() * wgt[w];         // dD/dV_al, conjugated
                }
                g[norb + nbath + l * norb + a] = tv * scale;
            }
            g[norb + l] = te * scale;
        }
        return g;
    }
};

// Minimiser of the cubic that matches value and slope at both ends of
// [lo, hi] (Hermite interpolation); NaN when that cubic has no interior minimum.
double cubic_step(double lo, double flo, double slo, double hi, double fhi, double shi)
{
    const double h = hi - lo;
    const double d1 = slo + shi - 3.0 * (fhi - flo) / h;
    const double disc = d1 * d1 - slo * shi;
    if (!(disc >= 0.0)) return NAN;
    const double d2 = std::copysign(std::sqrt(disc), h);
    const double den = shi - slo + 2.0 * d2;
    if (den == 0.0) return NAN;
    return hi - h * (shi + d2 - d1) / den;
}

struct LinePoint {
    double t, f, s;
};

// Minimum of phi(t) = f(p + t d) over t > 0 for a descent direction (slope
// s0 < 0 at t = 0), from values and slopes (phi(t, &slope) returns the value).
// Steps grow fourfold from t0 until the slope turns non-negative or the value
// rises above the last descending point's, which brackets a minimum; the
// bracket then shrinks around the Hermite-cubic minimiser of its ends, held to
// the middle 80% of the bracket (else its midpoint).  Stops when the slope has
// fallen below rtol |s0| or the bracket below rtol (|t| + rtol).  Returns the
// lowest point evaluated.  The same search as dmft.py's line_minimum.
template <class Phi>
LinePoint line_minimum(Phi& phi, double f0, double s0, double t0, double rtol = 1.0e-10, int maxeval = 200)
{
    LinePoint lo{0.0, f0, s0}, hi{0.0, 0.0, 0.0}, best = lo;
    bool have_hi = false;
    double t = t0;
    int n = 0;
    while (!have_hi) {
        double st = 0.0;
        const double ft = phi(t, &st);
        n++;
        if (!std::isfinite(ft) || !std::isfinite(st)) {
            hi = {t, INFINITY, INFINITY};
            have_hi = true;
            break;
        }
        if (ft < best.f) best = {t, ft, st};
        if (st >= 0.0 || ft > lo.f) {
            hi = {t, ft, st};
            have_hi = true;
            break;
        }
        lo = {t, ft, st};
        if (std::fabs(st) <= rtol * std::fabs(s0)) return best;
        if (n >= maxeval) throw Fail{EDZT_ERR_NUMERIC, "bath fit: line search found no bracket"};
        t *= 4.0;
    }
    while (n < maxeval) {
        const double w = hi.t - lo.t;
        if (w <= rtol * (std::fabs(lo.t) + rtol)) break;
        t = std::isfinite(hi.f) ? cubic_step(lo.t, lo.f, lo.s, hi.t, hi.f, hi.s) : NAN;
        if (!(t >= lo.t + 0.1 * w && t <= hi.t - 0.1 * w)) t = lo.t + 0.5 * w;
        double st = 0.0;
        const double ft = phi(t, &st);
        n++;
        if (ft < best.f) best = {t, ft, st};
        if (st < 0.0 && ft <= lo.f) lo = {t, ft, st};
        else hi = {t, ft, st};
        if (std::fabs(st) <= rtol * std::fabs(s0) && ft <= best.f) break;
    }
    return best;
}

double dot(const std::vector<double>& a, const std::vector<double>& b)
{
    double s = 0.0;
    for (size_t i = 0; i < a.size(); i++) s += a[i] * b[i];
    return s;
}

// Nonlinear conjugate gradient with Polak-Ribiere directions (the reference's
// fit method), restarted along the steepest descent when the update
// coefficient is negative or the direction does not descend, with
// line_minimum as the line search.  Stops when an iteration lowers f by no
// more than ftol relative to f, 2 (f_old - f_new) <= ftol (|f_old| + |f_new|
// + 1e-10 |f_start|), or when the gradient vanishes.  The same iteration as
// dmft.py's conjugate_gradient.
double conjugate_gradient(const BathFit& bf, std::vector<double>& p, double ftol, int* iters, int itmax = 20000)
{
    const size_t n = p.size();
    double fp = bf.f(p);
    const double floor = 1.0e-10 * std::fabs(fp);
    std::vector<double> g = bf.df(p), d(n), q(n);
    for (size_t i = 0; i < n; i++) d[i] = -g[i];
    double step = 1.0;
    for (int it = 1; it <= itmax; it++) {
        double s0 = dot(g, d);
        if (!(s0 < 0.0)) {                               // not a descent direction: restart
            for (size_t i = 0; i < n; i++) d[i] = -g[i];
            s0 = dot(g, d);
            if (!(s0 < 0.0)) { *iters = it; return fp; }
        }
        auto phi = [&](double t, double* slope) {
            for (size_t i = 0; i < n; i++) q[i] = p[i] + t * d[i];
            *slope = dot(bf.df(q), d);
            return bf.f(q);
        };
        const LinePoint lp = line_minimum(phi, fp, s0, step);
        for (size_t i = 0; i < n; i++) p[i] += lp.t * d[i];
        const std::vector<double> gn = bf.df(p);
        const double fn = lp.f;
        if (2.0 * (fp - fn) <= ftol * (std::fabs(fp) + std::fabs(fn) + floor)) {
            *iters = it;
            return fn;
        }
        double num = 0.0;
        for (size_t i = 0; i < n; i++) num += gn[i] * (gn[i] - g[i]);
        const double beta = std::max(0.0, num / dot(g, g));
        for (size_t i = 0; i < n; i++) d[i] = -gn[i] + beta * d[i];
        step = lp.t > 0.0 ? lp.t : 1.0;
        g = gn;
        fp = fn;
    }
    throw Fail{EDZT_ERR_NUMERIC, "bath fit: conjugate gradient did not converge"};
}

// New (em, ek, vmk), fitted per spin; with nspin 1 spin down copies spin up.
void fit_bath(int norb, int nbath, int nspin, int nw, const double* omega, double* em, double* ek, double* vmk,
              const cplx* D, const cplx* Gcl, const cplx* Gloc, double ftol, double* cost)
{
    for (int s = 0; s < nspin; s++) {
        BathFit bf(norb, nbath, nw, omega, em, D, Gcl, Gloc, s);
        std::vector<double> x(norb + nbath + norb * nbath);
        for (int a = 0; a < norb; a++) x[a] = em[a + norb * s];
        for (int l = 0; l < nbath; l++) x[norb + l] = ek[l + nbath * s];
        for (int l = 0; l < nbath; l++)
            for (int a = 0; a < norb; a++) x[norb + nbath + l * norb + a] = vmk[a + norb * (l + nbath * s)];
        int it = 0;
        const double fret = conjugate_gradient(bf, x, ftol, &it);
        if (cost) cost[s] = fret;
        for (int a = 0; a < norb; a++) em[a + norb * s] = x[a];
        for (int l = 0; l < nbath; l++) ek[l + nbath * s] = x[norb + l];
        for (int l = 0; l < nbath; l++)
            for (int a = 0; a < norb; a++) vmk[a + norb * (l + nbath * s)] = x[norb + nbath + l * norb + a];
    }
    if (nspin == 1) {
        for (int a = 0; a < norb; a++) em[a + norb] = em[a];
        for (int l = 0; l < nbath; l++) ek[l + nbath] = ek[l];
        for (int l = 0; l < nbath; l++)
            for (int a = 0; a < norb; a++) vmk[a + norb * (l + nbath)] = vmk[a + norb * l];
    }
}

// Each fitted bath site's couplings (the column vmk(:, l, s)) take the sign
// that best matches the previous ones.  The fit's cost depends on them only
// through products V_a V_b of one site, so a site's overall sign is free and
// the conjugate gradient may return either; linear mixing of vmk is only
// meaningful between columns of the same sign.
void align_bath_signs(int norb, int nbath, double* vmk_new, const double* vmk_old)
{
    for (int s = 0; s < 2; s++)
        for (int l = 0; l < nbath; l++) {
            double dot = 0.0;
            for (int a = 0; a < norb; a++) dot += vmk_new[a + norb * (l + nbath * s)] * vmk_old[a + norb * (l + nbath * s)];
            if (dot < 0.0)
                for (int a = 0; a < norb; a++) vmk_new[a + norb * (l + nbath * s)] = -vmk_new[a + norb * (l + nbath * s)];
        }
}

// ---- the reference's output files ------------------------------------------
std::string path_in(const char* dir, const std::string& name) { return std::string(dir) + "/" + name; }

void write_h_imp(const char* dir, int norb, int nbath, int nspin, const double* em, const double* ek,
                 const double* vmk)
{
    FILE* f = std::fopen(path_in(dir, "h_imp.dat").c_str(), "w");
    if (!f) throw Fail{EDZT_ERR_ARG, "cannot write an output file in outdir"};
    std::fprintf(f, " %11d %11d %11d\n", norb, nbath, nspin);
    for (int s = 0; s < nspin; s++) {
        for (int a = 0; a < norb; a++) std::fprintf(f, " %25.16E\n", em[a + norb * s]);
        for (int l = 0; l < nbath; l++) std::fprintf(f, " %25.16E\n", ek[l + nbath * s]);
        for (int l = 0; l < nbath; l++)
            for (int a = 0; a < norb; a++) std::fprintf(f, " %25.16E\n", vmk[a + norb * (l + nbath * s)]);
    }
    std::fclose(f);
}

// green.dat.<o>.<s> / sigma.dat.<o>.<s>: 'nw iorb ispin', then rows of w and
// the functions' real and imaginary parts in F12.8.
void write_functions(const char* dir, const char* stem, int norb, int nspin, int nw, const double* omega,
                     const std::vector<const cplx*>& fs)
{
    for (int s = 0; s < nspin; s++)
        for (int a = 0; a < norb; a++) {
            const std::string name = std::string(stem) + "." + std::to_string(a + 1) + "." + std::to_string(s + 1);
            FILE* f = std::fopen(path_in(dir, name).c_str(), "w");
            if (!f) throw Fail{EDZT_ERR_ARG, "cannot write an output file in outdir"};
            std::fprintf(f, " %11d %11d %11d\n", nw, a + 1, s + 1);
            for (int w = 0; w < nw; w++) {
                std::fprintf(f, "%12.8f", omega[w]);
                for (const cplx* F : fs) {
                    const cplx z = F[gidx(w, a, s, nw, norb)];
                    std::fprintf(f, "%12.8f%12.8f", z.real(), z.imag());
                }
                std::fprintf(f, "\n");
            }
            std::fclose(f);
        }
}

// g_coeffs.dat (dmft_green.f90:66-109): 'maxnstep norb', then per orbital and
// spin 1, 2 the line 'iorb ispin E0' and maxnstep rows of ap, bp, am, bm.
// coeffs: [norb][2][4][maxnstep] as edzt_cluster_green_ftn returns them.
void write_g_coeffs(const char* dir, int norb, int maxnstep, double e0, const double* coeffs)
{
    FILE* f = std::fopen(path_in(dir, "g_coeffs.dat").c_str(), "w");
    if (!f) throw Fail{EDZT_ERR_ARG, "cannot write an output file in outdir"};
    std::fprintf(f, " %11d %11d\n", maxnstep, norb);
    for (int a = 0; a < norb; a++)
        for (int s = 0; s < 2; s++) {
            std::fprintf(f, "%4d%4d %25.16E\n", a + 1, s + 1, e0);
            const double* c = coeffs + (size_t)(a * 2 + s) * 4 * maxnstep;
            for (int i = 0; i < maxnstep; i++)
                std::fprintf(f, "%25.16E %25.16E %25.16E %25.16E\n", c[i], c[maxnstep + i], c[2 * maxnstep + i],
                             c[3 * maxnstep + i]);
        }
    std::fclose(f);
}

bool finite_all(const double* p, size_t n)
{
    for (size_t i = 0; i < n; i++)
        if (!std::isfinite(p[i])) return false;
    return true;
}

}  // namespace

extern "C" {

int edzt_hybridization(int norb, int nbath, int nspin, int nw, const double* omega, const double* ek,
                       const double* vmk, double* D)
{
    if (norb < 1 || nbath < 0 || (nspin != 1 && nspin != 2) || nw < 1 || !omega || !D || (nbath > 0 && (!ek || !vmk)))
        return EDZT_ERR_ARG;
    hybridization(norb, nbath, nspin, nw, omega, ek, vmk, reinterpret_cast<cplx*>(D));
    return EDZT_OK;
}

int edzt_local_green_bethe(int norb, int nspin, int nw, const double* em, double hfield, const double* D,
                           const double* G_cl, double* G_loc)
{
    if (norb < 1 || (nspin != 1 && nspin != 2) || nw < 1 || !em || !D || !G_cl || !G_loc) return EDZT_ERR_ARG;
    local_green(norb, nspin, nw, em, hfield, reinterpret_cast<const cplx*>(D), reinterpret_cast<const cplx*>(G_cl),
                reinterpret_cast<cplx*>(G_loc));
    return EDZT_OK;
}

int edzt_fit_bath(int norb, int nbath, int nspin, int nw, const double* omega, double* em, double* ek, double* vmk,
                  const double* D, const double* G_cl, const double* G_loc, double ftol, double* cost)
{
    if (norb < 1 || nbath < 1 || (nspin != 1 && nspin != 2) || nw < 1 || !omega || !em || !ek || !vmk || !D ||
        !G_cl || !G_loc || !(ftol > 0.0))
        return EDZT_ERR_ARG;
    try {
        fit_bath(norb, nbath, nspin, nw, omega, em, ek, vmk, reinterpret_cast<const cplx*>(D),
                 reinterpret_cast<const cplx*>(G_cl), reinterpret_cast<const cplx*>(G_loc), ftol, cost);
    } catch (const Fail& e) {
        return e.code;
    }
    return EDZT_OK;
}

int edzt_dmft_bethe(edzt_ctx* ctx, const edzt_dmft_params* p, double* em, double* ek, double* vmk, double* D_cl,
                    double* G_cl, double* G_loc, double* Z, int* iterations, double* history, int* converged)
{
    if (!ctx || !p || !em || !ek || !vmk || !iterations || !converged) return EDZT_ERR_ARG;
    const int norb = p->norb, nbath = p->nbath, nspin = p->nspin, nw = p->nw;
    if (norb < 1 || nbath < 1 || (nspin != 1 && nspin != 2) || nw < 1 || !p->omega || p->nloop < 1 ||
        p->nsector < 1 || !p->sectors || p->maxnstep < 1 || !(p->mixing > 0.0 && p->mixing <= 1.0) ||
        !(p->fit_ftol > 0.0) || !finite_all(p->omega, nw)) {
        edzt_ctx_set_error(ctx, "edzt_dmft_bethe: invalid parameters (sizes, sectors, nloop, mixing in (0, 1], "
                                "fit_ftol > 0, finite omega)");
        return EDZT_ERR_ARG;
    }
    const size_t ng = (size_t)nw * norb * nspin;
    std::vector<cplx> D(ng), Gc(ng), Gl(ng);
    std::vector<double> coeffs((size_t)norb * 2 * 4 * p->maxnstep);
    *converged = 0;
    *iterations = 0;
    int rc = EDZT_OK;
    try {
        for (int it = 1; it <= p->nloop; it++) {
            if (it > 1) {                                         // dmft.f90:72-75
                std::vector<double> emf(em, em + 2 * norb), ekf(ek, ek + 2 * nbath),
                    vmf(vmk, vmk + 2 * (size_t)norb * nbath);
                fit_bath(norb, nbath, nspin, nw, p->omega, emf.data(), ekf.data(), vmf.data(), D.data(), Gc.data(),
                         Gl.data(), p->fit_ftol, nullptr);
                const double m = p->mixing;
                if (m < 1.0) align_bath_signs(norb, nbath, vmf.data(), vmk);
                for (int i = 0; i < 2 * norb; i++) em[i] = m * emf[i] + (1.0 - m) * em[i];
                for (int i = 0; i < 2 * nbath; i++) ek[i] = m * ekf[i] + (1.0 - m) * ek[i];
                for (size_t i = 0; i < 2 * (size_t)norb * nbath; i++) vmk[i] = m * vmf[i] + (1.0 - m) * vmk[i];
            }
            hybridization(norb, nbath, nspin, nw, p->omega, ek, vmk, D.data());
            if ((rc = edzt_set_model(ctx, norb, nbath, em, ek, vmk, p->U, p->Up, p->Jex, p->Jp, p->mu)) != EDZT_OK)
                throw Fail{rc, nullptr};
            int isector = 0;
            double e0 = 0.0;
            if ((rc = edzt_ground_state(ctx, p->nsector, p->sectors, p->maxnstep, p->seed, &isector, &e0, nullptr,
                                        nullptr)) != EDZT_OK)
                throw Fail{rc, nullptr};
            if ((rc = edzt_cluster_green_ftn(ctx, nspin, p->maxnstep, nw, p->omega, reinterpret_cast<double*>(Gc.data()),
                                             coeffs.data())) != EDZT_OK)
                throw Fail{rc, nullptr};
            local_green(norb, nspin, nw, em, p->hfield, D.data(), Gc.data(), Gl.data());
            if (p->outdir) {                                      // dump_data every iteration (dmft.f90:82)
                write_h_imp(p->outdir, norb, nbath, nspin, em, ek, vmk);
                write_functions(p->outdir, "green.dat", norb, nspin, nw, p->omega, {D.data(), Gc.data(), Gl.data()});
                write_g_coeffs(p->outdir, norb, p->maxnstep, e0, coeffs.data());
            }
            const double diff = scf_diff(norb, nbath, nspin, nw, Gc.data(), Gl.data());
            if (history) history[it - 1] = diff;
            *iterations = it;
            if (diff < p->scf_tol) { *converged = 1; break; }
        }
        // post_process: Sigma and Z
        std::vector<cplx> S(ng);
        for (int s = 0; s < nspin; s++)
            for (int a = 0; a < norb; a++)
                for (int w = 0; w < nw; w++) {
                    const size_t g = gidx(w, a, s, nw, norb);
                    S[g] = cplx(p->mu, p->omega[w]) - em[a + norb * s] - D[g] - 1.0 / Gc[g];
                }
        if (Z)
            for (int s = 0; s < nspin; s++)
                for (int a = 0; a < norb; a++)
                    Z[a + norb * s] = 1.0 / (1.0 - S[gidx(0, a, s, nw, norb)].imag() / p->omega[0]);
        if (p->outdir) write_functions(p->outdir, "sigma.dat", norb, nspin, nw, p->omega, {S.data()});
    } catch (const Fail& e) {
        if (e.msg) edzt_ctx_set_error(ctx, e.msg);
        return e.code;
    }
    if (D_cl) std::copy(D.begin(), D.end(), reinterpret_cast<cplx*>(D_cl));
    if (G_cl) std::copy(Gc.begin(), Gc.end(), reinterpret_cast<cplx*>(G_cl));
    if (G_loc) std::copy(Gl.begin(), Gl.end(), reinterpret_cast<cplx*>(G_loc));
    return EDZT_OK;
}

}  // extern "C"
