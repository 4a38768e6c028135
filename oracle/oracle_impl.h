/*
 * CPU restatement of the GBKFIT model-evaluation arithmetic.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is part of the oracle: it is compiled
 * into oracle/_build/liboracle.so and used by the test-suite, by smoke() and
 * by the CPU-baseline leg of bench.py as the checker.  The product path
 * (gbkfit_b200) never links, loads or calls it.
 *
 * The body is included twice by oracle.c, once with REAL=float (suffix _f32,
 * the reference's own precision) and once with REAL=double (suffix _f64, the
 * fp64 oracle).  <tgmath.h> makes sin/cos/... dispatch on REAL, mirroring the
 * reference's std:: overloads on T.
 *
 * Every function cites the reference file it restates; paths are relative to
 * src/gbkfit/driver/native/gbkfit/include/gbkfit/ unless stated otherwise.
 *
 * Deliberate divergences from the reference (all in degenerate cases that are
 * undefined behaviour there):
 *   - a spectral column whose line centre or width is not finite is skipped
 *     (gmodels.hpp:100-105 converts NaN to int, which is UB and on x86 writes
 *     out of bounds);
 *   - a cloud whose projected position is not finite is discarded
 *     (gmodels.hpp:499-508 converts NaN to int; on x86 that gives INT_MIN,
 *     which the bounds test then discards, so the result matches x86).
 */

#define CAT_(a, b) a##b
#define CAT(a, b) CAT_(a, b)
#define F(name) CAT(name, SFX)

#define R(x) ((REAL)(x))
#define PI_R R(3.14159265358979323846)
#define D2R (PI_R / R(180))

/* ---- math.hpp ---------------------------------------------------------- */

/* math.hpp:28-36 */
static REAL F(wrap_angle)(REAL a)
{
    while (a < -PI_R) a += 2 * PI_R;
    while (a > +PI_R) a -= 2 * PI_R;
    return a;
}

/* math.hpp:38-42 */
static int F(sgn)(REAL x) { return (R(0) < x) - (x < R(0)); }

/* math.hpp:44-51: left-handed rotation about x */
static void F(rot_lh_x)(REAL* oy, REAL* oz, REAL y, REAL z, REAL t)
{
    REAL s = sin(t), c = cos(t);
    *oy = y * c + z * s;
    *oz = -y * s + z * c;
}

/* math.hpp:62-71: the reference's (non-standard) left-handed z rotation */
static void F(rot_lh_z)(REAL* ox, REAL* oy, REAL x, REAL y, REAL t)
{
    REAL s = sin(t), c = cos(t);
    *ox = -x * s + y * c;
    *oy = -x * c - y * s;
}

/* math.hpp:126-143 */
static REAL F(uniform_fun)(REAL x, REAL a, REAL b, REAL c)
{ return x >= b && x <= c ? a : 0; }
static REAL F(uniform_cdf)(REAL x, REAL b, REAL c)
{ return x < b ? 0 : (x > c ? 1 : ((x - b) / (c - b))); }
static REAL F(uniform_pdf)(REAL x, REAL b, REAL c)
{ REAL a = 1 / (c - b); return F(uniform_fun)(x, a, b, c); }
/* math.hpp:164-193: "wm" = centre/half-width parametrisation */
static REAL F(uniform_wm_fun)(REAL x, REAL a, REAL b, REAL c)
{ return F(uniform_fun)(x, a, b - c, b + c); }
static REAL F(uniform_wm_pdf)(REAL x, REAL b, REAL c)
{ return F(uniform_pdf)(x, b - c, b + c); }
static REAL F(uniform_wm_pdf_trunc)(REAL x, REAL b, REAL c, REAL lo, REAL hi)
{
    return x >= lo && x <= hi
        ? F(uniform_pdf)(x, b - c, b + c)
          / (F(uniform_cdf)(hi, b - c, b + c) - F(uniform_cdf)(lo, b - c, b + c))
        : 0;
}

/* math.hpp:219-249 */
static REAL F(expon_fun)(REAL x, REAL a, REAL b, REAL c)
{ return a * exp(-fabs(x - b) / c); }
static REAL F(expon_cdf)(REAL x, REAL b, REAL c)
{ return R(0.5) + R(0.5) * F(sgn)(x - b) * (1 - exp(-fabs(x - b) / c)); }
static REAL F(expon_pdf)(REAL x, REAL b, REAL c)
{ REAL a = 1 / (2 * c); return F(expon_fun)(x, a, b, c); }

/* math.hpp:264-294 */
static REAL F(gauss_fun)(REAL x, REAL a, REAL b, REAL c)
{ return a * exp(-(x - b) * (x - b) / (2 * c * c)); }
static REAL F(gauss_cdf)(REAL x, REAL b, REAL c)
{ return (REAL)(0.5 * (1 + erf((double)(x - b) / ((double)c * sqrt(2.0))))); }
static REAL F(gauss_pdf)(REAL x, REAL b, REAL c)
{ REAL a = 1 / (c * sqrt(2 * PI_R)); return F(gauss_fun)(x, a, b, c); }

/* math.hpp:310-337 (the reference's ggauss cdf is a stub returning 0) */
static REAL F(ggauss_fun)(REAL x, REAL a, REAL b, REAL c, REAL d)
{ return a * exp(-pow(fabs(x - b) / c, d)); }
static REAL F(ggauss_cdf)(REAL x, REAL b, REAL c, REAL d)
{ (void)x; (void)b; (void)c; (void)d; return 0; }
static REAL F(ggauss_pdf)(REAL x, REAL b, REAL c, REAL d)
{ REAL a = d / (2 * c * tgamma(1 / d)); return F(ggauss_fun)(x, a, b, c, d); }

/* math.hpp:358-381 */
static REAL F(lorentz_fun)(REAL x, REAL a, REAL b, REAL c)
{ return a * c * c / ((x - b) * (x - b) + c * c); }
static REAL F(lorentz_cdf)(REAL x, REAL b, REAL c)
{ return R(0.5) + atan((x - b) / c) / PI_R; }
static REAL F(lorentz_pdf)(REAL x, REAL b, REAL c)
{ REAL a = 1 / (PI_R * c); return F(lorentz_fun)(x, a, b, c); }

/* math.hpp:403-434 (the reference's moffat cdf and pdf are stubs returning 0) */
static REAL F(moffat_fun)(REAL x, REAL a, REAL b, REAL c, REAL d)
{ return a / pow(1 + ((x - b) / c) * ((x - b) / c), d); }
static REAL F(moffat_cdf)(REAL x, REAL b, REAL c, REAL d)
{ (void)x; (void)b; (void)c; (void)d; return 0; }
static REAL F(moffat_pdf)(REAL x, REAL b, REAL c, REAL d)
{ (void)x; (void)b; (void)c; (void)d; return 0; }

/* math.hpp:455-478; std::pow(T, int) promotes to double in the reference */
static REAL F(sech2_fun)(REAL x, REAL a, REAL b, REAL c)
{ REAL q = 1 / cosh((x - b) / c); return (REAL)(a * ((double)q * (double)q)); }
static REAL F(sech2_cdf)(REAL x, REAL b, REAL c)
{ return R(0.5) * (1 + tanh((x - b) / c)); }
static REAL F(sech2_pdf)(REAL x, REAL b, REAL c)
{ REAL a = 1 / (2 * c); return F(sech2_fun)(x, a, b, c); }

/* math.hpp:108-114: truncated pdf = pdf / (cdf(hi) - cdf(lo)) on [lo, hi] */
#define TRUNC_PDF(pdf_expr, cdf_hi, cdf_lo, x, lo, hi) \
    ((x) >= (lo) && (x) <= (hi) ? (pdf_expr) / ((cdf_hi) - (cdf_lo)) : 0)
/* math.hpp:100-106 */
#define TRUNC_FUN(fun_expr, x, lo, hi) ((x) >= (lo) && (x) <= (hi) ? (fun_expr) : 0)

/* math.hpp:500-511 */
static REAL F(lerp)(REAL x, int idx, const REAL* xd, const REAL* yd, int off, int stride)
{
    REAL x1 = xd[idx - 1], x2 = xd[idx];
    REAL y1 = yd[off + (idx - 1) * stride], y2 = yd[off + idx * stride];
    REAL t = (x - x1) / (x2 - x1);
    return y1 + t * (y2 - y1);
}
#define NW(params, off) F(lerp)(r, rnidx, rnodes, (params), (off), 1)

/* ---- random numbers ---------------------------------------------------- */
/*
 * The reference draws from std::mt19937 seeded 42 in every OpenMP thread
 * (gbkfit_host/include/gbkfit/host/kernels.hpp:239-242), so its clouds depend
 * on the thread schedule and only statistical parity is possible.  Both this
 * oracle and the CUDA kernels instead use a counter-based Philox-4x32-10
 * stream keyed by (seed, cloud index): draw k of cloud ci is word (k % 4) of
 * Philox(counter = {ci, k / 4, 0, 0}, key = {seed_lo, seed_hi}).  Philox is
 * the published generator of Salmon et al., "Parallel random numbers: as easy
 * as 1, 2, 3" (SC'11).  A 32-bit word w maps to ((w >> 8) + 0.5) * 2^-24,
 * which lies strictly inside (0, 1).
 */
#ifndef ORACLE_PHILOX_DEFINED
#define ORACLE_PHILOX_DEFINED
typedef struct { unsigned ci; unsigned seed_lo, seed_hi; unsigned k; unsigned w[4]; } orc_rng;
static void orc_philox(const unsigned ctr_in[4], unsigned key0, unsigned key1, unsigned out[4])
{
    unsigned c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    unsigned k0 = key0, k1 = key1;
    for (int round = 0; round < 10; ++round) {
        unsigned long long p0 = (unsigned long long)0xD2511F53u * c0;
        unsigned long long p1 = (unsigned long long)0xCD9E8D57u * c2;
        unsigned hi0 = (unsigned)(p0 >> 32), lo0 = (unsigned)p0;
        unsigned hi1 = (unsigned)(p1 >> 32), lo1 = (unsigned)p1;
        unsigned n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}
static double orc_rng_next(orc_rng* g)
{
    if ((g->k & 3u) == 0) {
        unsigned ctr[4] = { g->ci, g->k >> 2, 0u, 0u };
        orc_philox(ctr, g->seed_lo, g->seed_hi, g->w);
    }
    unsigned w = g->w[g->k & 3u];
    g->k++;
    return ((double)(w >> 8) + 0.5) * (1.0 / 16777216.0);
}
#endif
#define RNG() ((REAL)orc_rng_next(rng))

/* ---- traits.hpp: polar traits ----------------------------------------- */

/* traits.hpp:199-246: blob mixtures; NP = 1 (6 params/blob) or 2 (7) */
static REAL F(p_mixture)(int kind, int np, REAL r, REAL theta, const REAL* consts, const REAL* params)
{
    REAL res = 0;
    int nb = (int)rint(consts[0]);
    for (int i = 0; i < nb; ++i) {
        REAL br = params[i], bt = params[1 * nb + i], ba = params[2 * nb + i];
        REAL bs = params[3 * nb + i];
        REAL bb = np == 2 ? params[4 * nb + i] : 0;
        REAL bq = params[(np == 2 ? 5 : 4) * nb + i];
        REAL bp = params[(np == 2 ? 6 : 5) * nb + i];
        bt *= D2R;
        bp *= D2R;
        REAL xn = r * cos(theta) - br * cos(bt);
        REAL yn = r * sin(theta) - br * sin(bt);
        F(rot_lh_z)(&xn, &yn, xn, yn, bt + bp);
        REAL rn = sqrt(xn * xn + (yn * yn) / (bq * bq));
        switch (kind) {
        case 51: res += F(expon_fun)(rn, ba, 0, bs); break;
        case 52: res += F(gauss_fun)(rn, ba, 0, bs); break;
        case 53: res += F(ggauss_fun)(rn, ba, 0, bs, bb); break;
        default: res += F(moffat_fun)(rn, ba, 0, bs, bb); break;
        }
    }
    return res;
}

/* traits.hpp:285-295 */
static REAL F(p_nw_harmonic)(int rnidx, const REAL* rnodes, int nrnodes, REAL r, REAL theta,
                             const REAL* consts, const REAL* params)
{
    int k = (int)rint(consts[0]);
    REAL a = NW(params, 0);
    REAL p = k ? NW(params, nrnodes) * D2R : 0;
    return a * cos(k * (theta - p));
}

/* traits.hpp:297-308 */
static REAL F(p_nw_distortion)(int rnidx, const REAL* rnodes, int nrnodes, REAL r, REAL theta,
                               const REAL* params)
{
    REAL a = NW(params, 0);
    REAL p = NW(params, nrnodes) * D2R;
    REAL s = NW(params, 2 * nrnodes);
    REAL t = F(wrap_angle)(theta - p);
    return a * exp(-(t * t * r * r) / (2 * s * s));
}

/* Shared body of the density (rp_trait, traits.hpp:1242-1331) and dispersion
 * (dp_trait, traits.hpp:1702-1775) polar traits, keyed by uid % 1000. */
static REAL F(p_profile)(int kind, const REAL* consts, const REAL* params,
                         int rnidx, const REAL* rnodes, int nrnodes, REAL r, REAL theta, int* err)
{
    switch (kind) {
    case 1: return params[0];
    case 2: return F(expon_fun)(r, params[0], 0, params[1]);
    case 3: return F(gauss_fun)(r, params[0], 0, params[1]);
    case 4: return F(ggauss_fun)(r, params[0], 0, params[1], params[2]);
    case 5: return F(lorentz_fun)(r, params[0], 0, params[1]);
    case 6: return F(moffat_fun)(r, params[0], 0, params[1], params[2]);
    case 7: return F(sech2_fun)(r, params[0], 0, params[1]);
    case 51: return F(p_mixture)(51, 1, r, theta, consts, params);
    case 52: return F(p_mixture)(52, 1, r, theta, consts, params);
    case 53: return F(p_mixture)(53, 2, r, theta, consts, params);
    case 54: return F(p_mixture)(54, 2, r, theta, consts, params);
    case 101: return NW(params, 0);
    case 102: return F(p_nw_harmonic)(rnidx, rnodes, nrnodes, r, theta, consts, params);
    case 103: return F(p_nw_distortion)(rnidx, rnodes, nrnodes, r, theta, params);
    default: *err = 1; return NAN;
    }
}

/* traits.hpp:1242-1331: surface-brightness (uid) and opacity (1000 + uid) */
static REAL F(rp_trait)(int uid, const REAL* c, const REAL* p, int rnidx, const REAL* rnodes,
                        int nrnodes, REAL r, REAL theta, int* err)
{
    int kind = uid >= 1000 ? uid - 1000 : uid;
    return F(p_profile)(kind, c, p, rnidx, rnodes, nrnodes, r, theta, err);
}

/* traits.hpp:1702-1775 */
static REAL F(dp_trait)(int uid, const REAL* c, const REAL* p, int rnidx, const REAL* rnodes,
                        int nrnodes, REAL r, REAL theta, int* err)
{
    return F(p_profile)(uid, c, p, rnidx, rnodes, nrnodes, r, theta, err);
}

/* traits.hpp:898-1078, 1592-1673: velocity polar traits */
static REAL F(vp_trait)(int uid, const REAL* consts, const REAL* params, int rnidx,
                        const REAL* rnodes, int nrnodes, REAL r, REAL theta, REAL incl, int* err)
{
    REAL out, rt = params[0], vt = uid >= 2 && uid <= 8 ? params[1] : 0;
    REAL mtan = cos(theta) * sin(incl);
    REAL mrad = sin(theta) * sin(incl);
    switch (uid) {
    case 1: out = params[0]; return out * mtan;
    case 2: out = vt * (2 / PI_R) * atan(r / rt); return out * mtan;
    case 3: out = vt * (1 - exp(-r / rt)); return out * mtan;
    case 4: out = vt * pow(r / rt, params[3]) / (1 + pow(r / rt, params[2])); return out * mtan;
    case 5: out = r < rt ? vt * r / rt : vt; return out * mtan;
    case 6: out = vt * tanh(r / rt); return out * mtan;
    case 7: out = vt * (1 - exp(-r / rt)) * (1 + params[2] * r / rt); return out * mtan;
    case 8: out = vt * pow(1 + r / rt, params[2]) * pow(1 + pow(r / rt, -params[3]), -1 / params[3]);
            return out * mtan;
    case 101: if (r == 0) return 0; out = NW(params, 0); return out * mtan;
    case 102: if (r == 0) return 0;
              out = F(p_nw_harmonic)(rnidx, rnodes, nrnodes, r, theta, consts, params);
              return out * mtan;
    case 103: if (r == 0) return 0; out = NW(params, 0); return out * mrad;
    case 104: if (r == 0) return 0;
              out = F(p_nw_harmonic)(rnidx, rnodes, nrnodes, r, theta, consts, params);
              return out * mrad;
    case 105: out = NW(params, 0); return out * cos(incl);
    case 106: out = F(p_nw_harmonic)(rnidx, rnodes, nrnodes, r, theta, consts, params);
              return out * cos(incl);
    case 107: return NW(params, 0);
    case 108: return F(p_nw_harmonic)(rnidx, rnodes, nrnodes, r, theta, consts, params);
    default: *err = 1; return NAN;
    }
}

/* traits.hpp:1177-1193, 1804-1829: vertical distortion */
static REAL F(zp_trait)(int uid, const REAL* c, const REAL* p, int rnidx, const REAL* rnodes,
                        int nrnodes, REAL r, REAL theta, int* err)
{
    if (uid == 101) return NW(p, 0);
    if (uid == 102) return F(p_nw_harmonic)(rnidx, rnodes, nrnodes, r, theta, c, p);
    *err = 1;
    return NAN;
}

/* traits.hpp:1195-1227 */
static REAL F(azrange)(REAL theta, REAL p, REAL s)
{
    REAL pmin = p - s * R(0.5);
    REAL pmax = p + s * R(0.5);
    pmin = F(wrap_angle)(pmin);
    pmax = F(wrap_angle)(pmax);
    if (pmin < pmax) return (theta > pmin && theta < pmax) ? 1 : 0;
    return (theta < pmin && theta > pmax) ? 0 : 1;
}

/* traits.hpp:1831-1857 */
static REAL F(sp_trait)(int uid, const REAL* c, const REAL* p, int rnidx, const REAL* rnodes,
                        int nrnodes, REAL r, REAL theta, int* err)
{
    (void)c;
    if (uid == 1) return F(azrange)(theta, p[0] * D2R, p[1] * D2R);
    if (uid == 101) return F(azrange)(theta, NW(p, 0) * D2R, NW(p, nrnodes) * D2R);
    *err = 1;
    return NAN;
}

/* traits.hpp:1229-1240, 1859-1885 (the reference's axis-range weight is a stub: 1) */
static REAL F(wp_trait)(int uid, int* err)
{
    if (uid == 1) return 1;
    *err = 1;
    return NAN;
}

/* ---- traits.hpp: height traits ----------------------------------------- */

/* traits.hpp:561-594, 633-896, 1437-1514 */
static REAL F(rh_trait)(int uid, const REAL* consts, const REAL* params, int rnidx,
                        const REAL* rnodes, int nrnodes, REAL r, REAL z, int* err)
{
    REAL trunc = consts[0];
    int use_rn = consts[1] != 0;
    REAL p1 = use_rn ? NW(params, 0) : params[0];
    if (uid >= 1 && uid <= 7) {
        /* surface brightness: pdfs (traits.hpp:561-594) */
        REAL p2 = (uid == 4 || uid == 6) ? (use_rn ? NW(params, nrnodes) : params[1]) : 0;
        REAL lo = -trunc * p1, hi = trunc * p1;
        switch (uid) {
        case 1: return trunc == 0 ? F(uniform_wm_pdf)(z, 0, p1)
                                  : F(uniform_wm_pdf_trunc)(z, 0, p1, lo, hi);
        case 2: return trunc == 0 ? F(expon_pdf)(z, 0, p1)
                : TRUNC_PDF(F(expon_pdf)(z, 0, p1), F(expon_cdf)(hi, 0, p1), F(expon_cdf)(lo, 0, p1), z, lo, hi);
        case 3: return trunc == 0 ? F(gauss_pdf)(z, 0, p1)
                : TRUNC_PDF(F(gauss_pdf)(z, 0, p1), F(gauss_cdf)(hi, 0, p1), F(gauss_cdf)(lo, 0, p1), z, lo, hi);
        case 4: return trunc == 0 ? F(ggauss_pdf)(z, 0, p1, p2)
                : TRUNC_PDF(F(ggauss_pdf)(z, 0, p1, p2), F(ggauss_cdf)(hi, 0, p1, p2), F(ggauss_cdf)(lo, 0, p1, p2), z, lo, hi);
        case 5: return trunc == 0 ? F(lorentz_pdf)(z, 0, p1)
                : TRUNC_PDF(F(lorentz_pdf)(z, 0, p1), F(lorentz_cdf)(hi, 0, p1), F(lorentz_cdf)(lo, 0, p1), z, lo, hi);
        case 6: return trunc == 0 ? F(moffat_pdf)(z, 0, p1, p2)
                : TRUNC_PDF(F(moffat_pdf)(z, 0, p1, p2), F(moffat_cdf)(hi, 0, p1, p2), F(moffat_cdf)(lo, 0, p1, p2), z, lo, hi);
        default: return trunc == 0 ? F(sech2_pdf)(z, 0, p1)
                : TRUNC_PDF(F(sech2_pdf)(z, 0, p1), F(sech2_cdf)(hi, 0, p1), F(sech2_cdf)(lo, 0, p1), z, lo, hi);
        }
    }
    if (uid >= 1001 && uid <= 1007) {
        /* opacity: unnormalised functions, amplitude first (traits.hpp:633-672);
         * the 3-parameter form reads params[1] for its third smooth parameter */
        REAL p2 = use_rn ? NW(params, nrnodes) : params[1];
        REAL p3 = use_rn ? NW(params, 2 * nrnodes) : params[1];
        REAL lo = -trunc * p2, hi = trunc * p2;
        REAL v;
        switch (uid - 1000) {
        case 1: v = F(uniform_wm_fun)(z, p1, 0, p2); break;
        case 2: v = F(expon_fun)(z, p1, 0, p2); break;
        case 3: v = F(gauss_fun)(z, p1, 0, p2); break;
        case 4: v = F(ggauss_fun)(z, p1, 0, p2, p3); break;
        case 5: v = F(lorentz_fun)(z, p1, 0, p2); break;
        case 6: v = F(moffat_fun)(z, p1, 0, p2, p3); break;
        default: v = F(sech2_fun)(z, p1, 0, p2); break;
        }
        return trunc == 0 ? v : TRUNC_FUN(v, z, lo, hi);
    }
    *err = 1;
    return NAN;
}

/* traits.hpp:1675-1700, 1777-1802: the only velocity/dispersion height trait */
static REAL F(one_trait)(int uid, int* err)
{
    if (uid == 1) return 1;
    *err = 1;
    return NAN;
}

/* ---- random sampling (mcdisk) ------------------------------------------ */

/* traits.hpp:310-326 */
static void F(sample_polar)(REAL* out_r, REAL* out_t, orc_rng* rng, REAL rmin, REAL rmax)
{
    REAL u1 = RNG();
    *out_r = sqrt(rmax * rmax + (rmin * rmin - rmax * rmax) * u1);
    REAL u2 = RNG();
    *out_t = 2 * PI_R * u2;
}
static void F(sample_polar_nw)(REAL* out_r, REAL* out_t, orc_rng* rng, int rnidx, const REAL* rnodes)
{
    REAL hw = rnodes[1] - rnodes[0];
    F(sample_polar)(out_r, out_t, rng, rnodes[rnidx] - hw, rnodes[rnidx] + hw);
}

/* traits.hpp:1333-1435; ridx is a ring index, rnidx = ridx + 1 its centre node */
static void F(rp_trait_rnd)(REAL* out_s, REAL* out_r, REAL* out_t, orc_rng* rng, int uid,
                            const REAL* consts, const REAL* params, int ridx,
                            const REAL* rnodes, int nrnodes, int* err)
{
    int rnidx = ridx + 1;
    int kind = uid >= 1000 ? uid - 1000 : uid;
    switch (kind) {
    case 1: F(sample_polar)(out_r, out_t, rng, rnodes[0], rnodes[nrnodes - 1]); break;
    case 2: case 3: case 4: case 5: case 6: case 7: case 101:
        F(sample_polar_nw)(out_r, out_t, rng, rnidx, rnodes); break;
    case 51: case 52: case 53: case 54: case 103:
        break; /* not implemented in the reference: outputs untouched */
    case 102: {
        F(sample_polar_nw)(out_r, out_t, rng, rnidx, rnodes);
        int k = (int)rint(consts[0]);
        REAL a = params[rnidx];
        REAL p = params[nrnodes + rnidx] * D2R;
        REAL vr = a * (RNG() * 2 - R(1));
        REAL vf = a * cos(k * (*out_t - p));
        *out_s = vr > vf ? 1 : -1;
        break;
    }
    default: *out_s = NAN; *out_r = NAN; *out_t = NAN; *err = 1; break;
    }
}

/* math.hpp:207-217: rejection sampling of a pdf on [-trunc, trunc] */
static REAL F(rejection)(int which, orc_rng* rng, REAL trunc, REAL b, REAL c, REAL d)
{
    REAL x, y, z;
    do {
        x = (0 - trunc) + RNG() * ((0 + trunc) - (0 - trunc));
        REAL u = RNG();
        y = (which == 4 ? F(ggauss_pdf)(0, b, c, d) : F(moffat_pdf)(0, b, c, d)) * u;
        z = which == 4 ? F(ggauss_pdf)(x, b, c, d) : F(moffat_pdf)(x, b, c, d);
    } while (y > z);
    return x;
}

/* math.hpp:152-498 sampling functions, selected as in traits.hpp:596-631 */
static REAL F(rnd_1d)(int kind, orc_rng* rng, REAL b, REAL c, REAL d)
{
    REAL u;
    switch (kind) {
    case 1: return (b - c) + RNG() * ((b + c) - (b - c));
    case 2: u = RNG() * 2 - R(1); return b - c * F(sgn)(u) * log(1 - 2 * fabs(u));
    case 3: { REAL u1 = RNG(); REAL u2 = RNG();
              return b + c * sqrt(-2 * log(u1)) * cos(2 * PI_R * u2); }
    case 4: return F(rejection)(4, rng, 5 * c, b, c, d);
    case 5: u = RNG() * 2 - R(1); return b + c * tan(PI_R * R(0.5) * u);
    case 6: return F(rejection)(6, rng, 5 * c, b, c, d);
    default: u = RNG() * 2 - R(1); return b + c * atanh(u);
    }
}

/* traits.hpp:596-631, 1516-1590 */
static REAL F(rh_trait_rnd)(orc_rng* rng, int uid, const REAL* consts, const REAL* params,
                            int rnidx, const REAL* rnodes, int nrnodes, REAL r, int* err)
{
    int off = uid >= 1000 ? 1 : 0;
    int kind = uid - 1000 * off;
    if (kind < 1 || kind > 7) { *err = 1; return NAN; }
    REAL trunc = consts[0];
    int use_rn = consts[1] != 0;
    REAL p1 = use_rn ? NW(params, (off + 0) * nrnodes) : params[off + 0];
    REAL p2 = 0;
    if (kind == 4 || kind == 6)
        p2 = use_rn ? NW(params, (off + 1) * nrnodes) : params[off + 1];
    /* _trunc_1d_rnd (math.hpp:116-124) loops while (x < lo && x > hi), which
     * is never true, so the truncated and plain samplers draw the same value */
    (void)trunc;
    return F(rnd_1d)(kind, rng, 0, p1, p2);
}

/* ---- gmodels.hpp -------------------------------------------------------- */

/* gmodels.hpp:92-116: Gaussian line (pdf, not multiplied by the channel
 * width) added to channels rint((v -+ 5 sigma - zero) / step), clamped */
static void F(splat_line)(REAL* scube, int x, int y, REAL rv, REAL vv, REAL dv,
                          int nx, int ny, int nz, REAL step, REAL zero)
{
    if (!isfinite(vv) || !isfinite(dv)) return;
    REAL zmin = vv - dv * 5, zmax = vv + dv * 5;
    REAL a = rint((zmin - zero) / step), b = rint((zmax - zero) / step);
    int zlo = (int)(a < 0 ? 0 : a);
    int zhi = (int)((REAL)(nz - 1) < b ? (REAL)(nz - 1) : b);
    for (int z = zlo; z <= zhi; ++z) {
        REAL zv = zero + z * step;
        scube[x + (long)nx * (y + (long)ny * z)] += rv * F(gauss_pdf)(zv, vv, dv);
    }
}

/* gmodels.hpp:197-215: linear search of the radial nodes */
static int F(disk_info)(int* idx, REAL r, int n, const REAL* nodes)
{
    if (r < nodes[0]) return 0;
    if (r >= nodes[n - 1]) return 0;
    for (*idx = 1; *idx < n; ++*idx)
        if (r < nodes[*idx]) break;
    return 1;
}

/* gmodels.hpp:118-195: sky <-> disk transforms */
static void F(cpos_posa_incl_2d)(REAL* x, REAL* y, REAL xp, REAL yp, REAL pa, REAL in)
{
    *x -= xp; *y -= yp;
    F(rot_lh_z)(x, y, *x, *y, pa);
    *y /= cos(in);
}
static void F(cpos_posa_incl_3d)(REAL* x, REAL* y, REAL* z, REAL xp, REAL yp, REAL pa, REAL in)
{
    *x -= xp; *y -= yp;
    F(rot_lh_z)(x, y, *x, *y, pa);
    F(rot_lh_x)(y, z, *y, *z, in);
}
static REAL F(rnode_radius)(REAL x, REAL y, REAL z, int thick, int loose, int tilted, int i,
                            const REAL* xpos, const REAL* ypos, const REAL* posa, const REAL* incl)
{
    REAL xp = loose ? xpos[i] : xpos[0], yp = loose ? ypos[i] : ypos[0];
    REAL pa = tilted ? posa[i] : posa[0], in = tilted ? incl[i] : incl[0];
    pa *= D2R; in *= D2R;
    if (thick) F(cpos_posa_incl_3d)(&x, &y, &z, xp, yp, pa, in);
    else F(cpos_posa_incl_2d)(&x, &y, xp, yp, pa, in);
    return sqrt(x * x + y * y);
}

/* gmodels.hpp:217-323: per-node re-projection search, "velfi" radius */
static int F(ring_info)(int* index, REAL* radius, REAL x, REAL y, REAL z, int thick, int loose,
                        int tilted, int n, const REAL* nodes, const REAL* xpos,
                        const REAL* ypos, const REAL* posa, const REAL* incl)
{
#define RR(i) F(rnode_radius)(x, y, z, thick, loose, tilted, (i), xpos, ypos, posa, incl)
    if (RR(0) < nodes[0]) return 0;
    if (RR(n - 1) >= nodes[n - 1]) return 0;
    for (*index = 1; *index < n; ++*index)
        if (RR(*index) < nodes[*index]) break;
    REAL d1 = nodes[*index - 1] - RR(*index - 1);
    REAL d2 = nodes[*index] - RR(*index);
    *radius = (nodes[*index] * d1 - nodes[*index - 1] * d2) / (d1 - d2);
    return 1;
#undef RR
}

/* The per-call trait tables, in the order of the reference's argument list */
typedef struct {
    int n;
    const int* uids; const REAL* cv; const int* cc; const REAL* pv; const int* pc;
} F(tset);

/* traits.hpp:1887-1919: evaluate every trait of a set, advancing the
 * constants/parameters pointers by the per-trait counts */
#ifndef ORACLE_KINDS_DEFINED
#define ORACLE_KINDS_DEFINED
enum { K_RP, K_RH, K_VP, K_VH, K_DP, K_DH, K_ZP, K_SP, K_WP };
#endif
static void F(eval_set)(REAL* out, int kind, int n, const int* uids, const REAL* cv, const int* cc,
                        const REAL* pv, const int* pc, int rnidx, const REAL* rnodes, int nrnodes,
                        REAL r, REAL theta, REAL incl, REAL z, int* err)
{
    for (int i = 0; i < n; ++i) {
        switch (kind) {
        case K_RP: out[i] = F(rp_trait)(uids[i], cv, pv, rnidx, rnodes, nrnodes, r, theta, err); break;
        case K_RH: out[i] = F(rh_trait)(uids[i], cv, pv, rnidx, rnodes, nrnodes, r, z, err); break;
        case K_VP: out[i] = F(vp_trait)(uids[i], cv, pv, rnidx, rnodes, nrnodes, r, theta, incl, err); break;
        case K_VH: case K_DH: out[i] = F(one_trait)(uids[i], err); break;
        case K_DP: out[i] = F(dp_trait)(uids[i], cv, pv, rnidx, rnodes, nrnodes, r, theta, err); break;
        case K_ZP: out[i] = F(zp_trait)(uids[i], cv, pv, rnidx, rnodes, nrnodes, r, theta, err); break;
        case K_SP: out[i] = F(sp_trait)(uids[i], cv, pv, rnidx, rnodes, nrnodes, r, theta, err); break;
        default: out[i] = F(wp_trait)(uids[i], err); break;
        }
        cv += cc[i];
        pv += pc[i];
    }
}

/* Argument bundle for one smdisk/mcdisk call (the reference passes these as
 * ~90 separate arguments, host/include/gbkfit/host/gmodels.hpp:26-135). */
typedef struct {
    int loose, tilted, nrnodes;
    const REAL *rnodes, *vsys, *xpos, *ypos, *posa, *incl;
    int nrt; const int* rpt_uids; const REAL* rpt_cv; const int* rpt_cc; const REAL* rpt_pv; const int* rpt_pc;
    const int* rht_uids; const REAL* rht_cv; const int* rht_cc; const REAL* rht_pv; const int* rht_pc;
    int nvt; const int* vpt_uids; const REAL* vpt_cv; const int* vpt_cc; const REAL* vpt_pv; const int* vpt_pc;
    const int* vht_uids; const REAL* vht_cv; const int* vht_cc; const REAL* vht_pv; const int* vht_pc;
    int ndt; const int* dpt_uids; const REAL* dpt_cv; const int* dpt_cc; const REAL* dpt_pv; const int* dpt_pc;
    const int* dht_uids; const REAL* dht_cv; const int* dht_cc; const REAL* dht_pv; const int* dht_pc;
    int nzt; const int* zpt_uids; const REAL* zpt_cv; const int* zpt_cc; const REAL* zpt_pv; const int* zpt_pc;
    int nst; const int* spt_uids; const REAL* spt_cv; const int* spt_cc; const REAL* spt_pv; const int* spt_pc;
    int nwt; const int* wpt_uids; const REAL* wpt_cv; const int* wpt_cc; const REAL* wpt_pv; const int* wpt_pc;
    const REAL* opacity;
    int sx, sy, sz; REAL stx, sty, stz; REAL zx, zy, zz;
    int spec_size; REAL spec_step, spec_zero;
    REAL *image, *scube, *wdata, *wdata_cmp, *rdata, *rdata_cmp, *ordata, *ordata_cmp, *vdata_cmp, *ddata_cmp;
} F(disk_args);

#define SET(a, pfx) a->pfx##_uids, a->pfx##_cv, a->pfx##_cc, a->pfx##_pv, a->pfx##_pc

/* gmodels.hpp:645-958: one spaxel (x, y, z) of the spatial grid */
static void F(smdisk_spaxel)(const F(disk_args)* a, int x, int y, int z, int* err)
{
    int thin = a->rht_uids == NULL;
    int rnidx = -1;
    REAL rn = 0, theta;
    REAL xn = a->zx + x * a->stx, yn = a->zy + y * a->sty, zn = a->zz + z * a->stz;
    const REAL* rnodes = a->rnodes;
    int nrn = a->nrnodes;
    if (a->loose || a->tilted) {
        if (!F(ring_info)(&rnidx, &rn, xn, yn, zn, !thin, a->loose, a->tilted, nrn, rnodes,
                          a->xpos, a->ypos, a->posa, a->incl))
            return;
    }
    /* gmodels.hpp:726: the loose systemic velocity interpolates xpos */
    REAL vsysi = a->loose ? F(lerp)(rn, rnidx, rnodes, a->xpos, 0, 1) : (a->vsys ? a->vsys[0] : 0);
    REAL xposi = a->loose ? F(lerp)(rn, rnidx, rnodes, a->xpos, 0, 1) : a->xpos[0];
    REAL yposi = a->loose ? F(lerp)(rn, rnidx, rnodes, a->ypos, 0, 1) : a->ypos[0];
    REAL posai = a->tilted ? F(lerp)(rn, rnidx, rnodes, a->posa, 0, 1) : a->posa[0];
    REAL incli = a->tilted ? F(lerp)(rn, rnidx, rnodes, a->incl, 0, 1) : a->incl[0];
    posai *= D2R;
    incli *= D2R;
    if (thin) F(cpos_posa_incl_2d)(&xn, &yn, xposi, yposi, posai, incli);
    else F(cpos_posa_incl_3d)(&xn, &yn, &zn, xposi, yposi, posai, incli);
    theta = atan2(yn, xn);
    if (!(a->loose || a->tilted)) {
        rn = sqrt(xn * xn + yn * yn);
        if (!F(disk_info)(&rnidx, rn, nrn, rnodes)) return;
    }
    REAL pt[4] = {0, 0, 0, 0}, ht[4] = {0, 0, 0, 0};
    REAL rv = 0, vv = 0, dv = 0, zv = 0, sv = 0, wv = 1;
    REAL r = rn;
    if (a->spt_uids) {
        F(eval_set)(pt, K_SP, a->nst, SET(a, spt), rnidx, rnodes, nrn, r, theta, 0, 0, err);
        for (int i = 0; i < a->nst; ++i) sv += pt[i];
        if (!sv) return;
    }
    if (a->zpt_uids) {
        F(eval_set)(pt, K_ZP, a->nzt, SET(a, zpt), rnidx, rnodes, nrn, r, theta, 0, 0, err);
        for (int i = 0; i < a->nzt; ++i) zv += pt[i];
        zn += zv;
    }
    if (a->rpt_uids)
        F(eval_set)(pt, K_RP, a->nrt, SET(a, rpt), rnidx, rnodes, nrn, r, theta, 0, 0, err);
    if (a->rht_uids)
        F(eval_set)(ht, K_RH, a->nrt, SET(a, rht), rnidx, rnodes, nrn, r, theta, 0, fabs(zn), err);
    for (int i = 0; i < a->nrt; ++i) rv += pt[i] * (thin ? 1 : ht[i]);
    if (!rv) return;
    if (thin) rv /= cos(incli);
    if (!thin) rv *= a->stz;
    if (a->vpt_uids)
        F(eval_set)(pt, K_VP, a->nvt, SET(a, vpt), rnidx, rnodes, nrn, r, theta, incli, 0, err);
    if (a->vht_uids)
        F(eval_set)(ht, K_VH, a->nvt, SET(a, vht), rnidx, rnodes, nrn, r, theta, 0, fabs(zn), err);
    for (int i = 0; i < a->nvt; ++i) vv += pt[i] * (thin ? 1 : ht[i]);
    vv += vsysi;
    if (a->dpt_uids)
        F(eval_set)(pt, K_DP, a->ndt, SET(a, dpt), rnidx, rnodes, nrn, r, theta, 0, 0, err);
    if (a->dht_uids)
        F(eval_set)(ht, K_DH, a->ndt, SET(a, dht), rnidx, rnodes, nrn, r, theta, 0, fabs(zn), err);
    for (int i = 0; i < a->ndt; ++i) dv += pt[i] * (thin ? 1 : ht[i]);
    dv = fabs(dv);
    if (a->wpt_uids && a->wdata) {
        F(eval_set)(pt, K_WP, a->nwt, SET(a, wpt), rnidx, rnodes, nrn, r, theta, 0, 0, err);
        for (int i = 0; i < a->nwt; ++i) wv *= pt[i];
    }
    REAL orv = rv;
    long sxy = (long)a->sx * a->sy;
    if (a->opacity)
        for (int oz = z + 1; oz < a->sz; ++oz)
            orv -= orv * a->opacity[x + (long)a->sx * y + sxy * oz];
    if (a->image) a->image[x + (long)a->sx * y] += orv;
    if (a->scube)
        F(splat_line)(a->scube, x, y, orv, vv, dv, a->sx, a->sy, a->spec_size, a->spec_step, a->spec_zero);
    long idx = x + (long)a->sx * y + sxy * z;
    if (a->wdata) a->wdata[idx] += wv;
    if (a->wdata_cmp) a->wdata_cmp[idx] = wv;
    if (a->rdata) a->rdata[idx] += rv;
    if (a->rdata_cmp) a->rdata_cmp[idx] = rv;
    if (a->ordata) a->ordata[idx] += orv;
    if (a->ordata_cmp) a->ordata_cmp[idx] = orv;
    if (a->vdata_cmp) a->vdata_cmp[idx] = vv;
    if (a->ddata_cmp) a->ddata_cmp[idx] = dv;
}

/* host/kernels.hpp:308-423: every spaxel of the spatial grid, sequentially */
static int F(smdisk_run)(const F(disk_args)* a)
{
    int err = 0;
    for (int y = 0; y < a->sy; ++y)
        for (int x = 0; x < a->sx; ++x)
            for (int z = 0; z < a->sz; ++z)
                F(smdisk_spaxel)(a, x, y, z, &err);
    return err;
}

/* gmodels.hpp:325-643: one Monte-Carlo cloud */
static void F(mcdisk_cloud)(const F(disk_args)* a, orc_rng* rng, int ci, REAL cflux,
                            const int* csum, const unsigned char* hasordint, int* err)
{
    const REAL* rnodes = a->rnodes;
    int nrn = a->nrnodes;
    int rnidx = 0, tidx;
    const REAL *rpc = a->rpt_cv, *rpp = a->rpt_pv, *rhc = a->rht_cv, *rhp = a->rht_pv;
    REAL xd, yd, zd = 0, rd = 0, theta = 0, sign = 1;
    REAL pt[4] = {0, 0, 0, 0}, ht[4] = {0, 0, 0, 0};
    REAL vv = 0, dv = 0, zv = 0, sv = 0, wv = 1;
    REAL rv = cflux / a->stz;
    while (ci >= csum[rnidx]) rnidx++;
    for (tidx = 0; tidx < a->nrt; ++tidx) {
        int size = hasordint[tidx] ? 1 : nrn - 2;
        if (rnidx < size) break;
        rnidx -= size;
        rpc += a->rpt_cc[tidx]; rpp += a->rpt_pc[tidx];
        rhc += a->rht_cc[tidx]; rhp += a->rht_pc[tidx];
    }
    F(rp_trait_rnd)(&sign, &rd, &theta, rng, a->rpt_uids[tidx], rpc, rpp, rnidx, rnodes, nrn, err);
    if (sign < 0) rv = -rv;
    rv *= a->stz;
    rv /= a->stx * a->sty;
    xd = rd * cos(theta);
    yd = rd * sin(theta);
    if (!F(disk_info)(&rnidx, rd, nrn, rnodes)) return;
    REAL r = rd;
    if (a->spt_uids) {
        F(eval_set)(pt, K_SP, a->nst, SET(a, spt), rnidx, rnodes, nrn, r, theta, 0, 0, err);
        for (int i = 0; i < a->nst; ++i) sv += pt[i];
        if (!sv) return;
    }
    zd = F(rh_trait_rnd)(rng, a->rht_uids[tidx], rhc, rhp, rnidx, rnodes, nrn, rd, err);
    if (a->zpt_uids) {
        F(eval_set)(pt, K_ZP, a->nzt, SET(a, zpt), rnidx, rnodes, nrn, r, theta, 0, 0, err);
        for (int i = 0; i < a->nzt; ++i) zv += pt[i];
        zd += zv;
    }
    REAL vsysi = a->vsys ? (a->loose ? F(lerp)(rd, rnidx, rnodes, a->vsys, 0, 1) : a->vsys[0]) : 0;
    REAL xposi = a->loose ? F(lerp)(rd, rnidx, rnodes, a->xpos, 0, 1) : a->xpos[0];
    REAL yposi = a->loose ? F(lerp)(rd, rnidx, rnodes, a->ypos, 0, 1) : a->ypos[0];
    REAL posai = a->tilted ? F(lerp)(rd, rnidx, rnodes, a->posa, 0, 1) : a->posa[0];
    REAL incli = a->tilted ? F(lerp)(rd, rnidx, rnodes, a->incl, 0, 1) : a->incl[0];
    posai *= D2R;
    incli *= D2R;
    /* gmodels.hpp:159-165 with negated parameters (gmodels.hpp:495-496) */
    REAL xn = xd, yn = yd, zn = zd;
    F(rot_lh_x)(&yn, &zn, yn, zn, -incli);
    F(rot_lh_z)(&xn, &yn, xn, yn, -posai);
    xn -= -xposi;
    yn -= -yposi;
    REAL fx = rint((xn - a->zx) / a->stx), fy = rint((yn - a->zy) / a->sty);
    REAL fz = rint((zn - a->zz) / a->stz);
    if (!isfinite(fx) || !isfinite(fy) || !isfinite(fz)) return;
    if (fx < 0 || fx >= a->sx || fy < 0 || fy >= a->sy || fz < 0 || fz >= a->sz) return;
    int x = (int)fx, y = (int)fy, z = (int)fz;
    if (a->vpt_uids)
        F(eval_set)(pt, K_VP, a->nvt, SET(a, vpt), rnidx, rnodes, nrn, r, theta, incli, 0, err);
    if (a->vht_uids)
        F(eval_set)(ht, K_VH, a->nvt, SET(a, vht), rnidx, rnodes, nrn, r, theta, 0, fabs(zd), err);
    for (int i = 0; i < a->nvt; ++i) vv += pt[i] * ht[i];
    vv += vsysi;
    if (a->dpt_uids)
        F(eval_set)(pt, K_DP, a->ndt, SET(a, dpt), rnidx, rnodes, nrn, r, theta, 0, 0, err);
    if (a->dht_uids)
        F(eval_set)(ht, K_DH, a->ndt, SET(a, dht), rnidx, rnodes, nrn, r, theta, 0, fabs(zd), err);
    for (int i = 0; i < a->ndt; ++i) dv += pt[i] * ht[i];
    dv = fabs(dv);
    if (a->wpt_uids && a->wdata) {
        F(eval_set)(pt, K_WP, a->nwt, SET(a, wpt), rnidx, rnodes, nrn, r, theta, 0, 0, err);
        for (int i = 0; i < a->nwt; ++i) wv *= pt[i];
    }
    REAL orv = rv;
    long sxy = (long)a->sx * a->sy;
    if (a->opacity)
        for (int oz = z + 1; oz < a->sz; ++oz)
            orv -= orv * a->opacity[x + (long)a->sx * y + sxy * oz];
    if (a->image) a->image[x + (long)a->sx * y] += orv;
    if (a->scube)
        F(splat_line)(a->scube, x, y, orv, vv, dv, a->sx, a->sy, a->spec_size, a->spec_step, a->spec_zero);
    long idx = x + (long)a->sx * y + sxy * z;
    if (a->wdata) a->wdata[idx] = wv;
    if (a->wdata_cmp) a->wdata_cmp[idx] = wv;
    if (a->rdata) a->rdata[idx] += rv;
    if (a->rdata_cmp) a->rdata_cmp[idx] += rv;
    if (a->ordata) a->ordata[idx] += orv;
    if (a->ordata_cmp) a->ordata_cmp[idx] += orv;
    if (a->vdata_cmp) a->vdata_cmp[idx] = vv;
    if (a->ddata_cmp) a->ddata_cmp[idx] = dv;
}

/* host/kernels.hpp:183-306, clouds in index order */
static int F(mcdisk_run)(const F(disk_args)* a, REAL cflux, int nclouds, const int* csum,
                         const unsigned char* hasordint, unsigned long long seed)
{
    int err = 0;
    for (int ci = 0; ci < nclouds; ++ci) {
        orc_rng g;
        g.ci = (unsigned)ci; g.seed_lo = (unsigned)seed; g.seed_hi = (unsigned)(seed >> 32);
        g.k = 0;
        F(mcdisk_cloud)(a, &g, ci, cflux, csum, hasordint, &err);
    }
    return err;
}

/* ---- dmodels.hpp, objective.hpp, host/kernels.hpp ------------------------ */

/* dmodels.hpp:7-46 */
void F(orc_dcube_downscale)(int scx, int scy, int scz, int ofx, int ofy, int ofz,
                            int srx, int sry, int srz, int dsx, int dsy, int dsz,
                            const REAL* src, REAL* dst)
{
    (void)srz;
    REAL nf = R(1) / (scx * scy * scz);
    for (int z = 0; z < dsz; ++z)
        for (int y = 0; y < dsy; ++y)
            for (int x = 0; x < dsx; ++x) {
                int nx = ofx + x * scx, ny = ofy + y * scy, nz = ofz + z * scz;
                REAL sum = 0;
                for (int dz = 0; dz < scz; ++dz)
                    for (int dy = 0; dy < scy; ++dy)
                        for (int dx = 0; dx < scx; ++dx)
                            sum += src[(nx + dx) + (long)srx * ((ny + dy) + (long)sry * (nz + dz))];
                dst[x + (long)dsx * (y + (long)dsy * z)] = sum * nf;
            }
}

/* dmodels.hpp:48-74 */
void F(orc_dcube_mask)(REAL cutoff, int apply, int nx, int ny, int nz, REAL* d, REAL* m, REAL* w)
{
    (void)w;
    long n = (long)nx * ny * nz;
    for (long i = 0; i < n; ++i) {
        REAL mv = 1;
        if (fabs(d[i]) <= cutoff) { mv = 0; if (apply) d[i] = NAN; }
        if (m) m[i] = mv;
    }
}

/* dmodels.hpp:76-228 for one pixel; mmaps_m receives the mask map and
 * mmaps_w the weight map (the template's own parameter names) */
static void F(moments_pixel)(int x, int y, int nx, int ny, int nz, REAL stz, REAL zz,
                             const REAL* d, const REAL* w, REAL cutoff, int norders,
                             const int* orders, REAL* md, REAL* mm, REAL* mw)
{
    long i2 = x + (long)nx * y, sxy = (long)nx * ny;
    int maxo = orders[norders - 1];
    int m = 0;
    REAL m0s = 0;
    for (int z = 0; z < nz; ++z) m0s += d[i2 + sxy * z] * stz;
    int valid = fabs(m0s) > cutoff;
    mm[i2] = (REAL)valid;
    REAL m0 = valid ? m0s : NAN;
    if (orders[m] == 0) { md[i2 + sxy * m] = m0; m++; }
    REAL ws = 0;
    for (int z = 0; w && valid && z < nz; ++z) ws += w[i2 + sxy * z] * d[i2 + sxy * z] * stz / m0;
    ws = valid ? ws : NAN;
    if (w) mw[i2] = ws;
    if (maxo == 0) return;
    REAL m1s = 0;
    for (int z = 0; valid && z < nz; ++z) m1s += d[i2 + sxy * z] * (zz + z * stz) * stz;
    REAL m1 = valid ? m1s / m0 : NAN;
    if (orders[m] == 1) { md[i2 + sxy * m] = m1; m++; }
    if (maxo == 1) return;
    REAL m2s = 0;
    for (int z = 0; valid && z < nz; ++z) {
        double dv = (double)((zz + z * stz) - m1);
        m2s = (REAL)((double)m2s + (double)d[i2 + sxy * z] * (dv * dv) * (double)stz);
    }
    REAL m2 = valid ? sqrt(m2s / m0) : NAN;
    if (orders[m] == 2) { md[i2 + sxy * m] = m2; m++; }
    for (; m < norders; ++m) {
        REAL mns = 0;
        for (int z = 0; valid && z < nz; ++z)
            mns = (REAL)((double)mns
                         + (double)d[i2 + sxy * z] * pow((double)((zz + z * stz) - m1), orders[m]));
        md[i2 + sxy * m] = valid ? mns / m0 : NAN;
    }
}

/* host/kernels.hpp:105-135 */
void F(orc_mmaps_moments)(int nx, int ny, int nz, REAL stx, REAL sty, REAL stz,
                          REAL zx, REAL zy, REAL zz, const REAL* d, const REAL* w, REAL cutoff,
                          int norders, const int* orders, REAL* mmaps_d, REAL* mmaps_m,
                          REAL* mmaps_w)
{
    (void)stx; (void)sty; (void)zx; (void)zy;
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x)
            F(moments_pixel)(x, y, nx, ny, nz, stz, zz, d, w, cutoff, norders, orders,
                             mmaps_d, mmaps_m, mmaps_w);
}

/* objective.hpp:7-31 */
void F(orc_residual)(const REAL* od, const REAL* oe, const REAL* om, const REAL* md,
                     const REAL* mw, const REAL* mm, long n, REAL weight, REAL* res)
{
    for (long i = 0; i < n; ++i) {
        REAL r = md[i] - od[i];
        if (oe) r /= oe[i];
        if (mw) r *= mw[i];
        if (om) r *= om[i];
        if (mm) r *= mm[i];
        res[i] = r * weight;
    }
}

/* host/kernels.hpp:502-514, accumulated in double */
double F(orc_residual_sum)(const REAL* res, long n, int squared)
{
    double s = 0;
    for (long i = 0; i < n; ++i) s += squared ? (double)res[i] * res[i] : fabs((double)res[i]);
    return s;
}

/* gmodels.hpp:52-82 */
void F(orc_wcube_evaluate)(int sx, int sy, int sz, int spec_z, const REAL* spat, REAL* spec)
{
    for (int y = 0; y < sy; ++y)
        for (int x = 0; x < sx; ++x) {
            REAL sum = 0, mx = 0;
            for (int z = 0; z < sz; ++z) {
                REAL v = spat[x + (long)sx * (y + (long)sy * z)];
                sum += v;
                mx = mx > v ? mx : v;
            }
            REAL mean = sum / sz;
            for (int z = 0; z < spec_z; ++z)
                spec[x + (long)sx * (y + (long)sy * z)] = mx > 0 ? mean / mx : 0;
        }
}

/* gmodels.hpp:9-50: direct (zero-padded) 3-D convolution */
void F(orc_convolve)(int ax, int ay, int az, int bx, int by, int bz, const REAL* a, const REAL* b,
                     REAL* out)
{
    for (int z = 0; z < az; ++z)
        for (int y = 0; y < ay; ++y)
            for (int x = 0; x < ax; ++x) {
                REAL s = 0;
                for (int z2 = 0; z2 < bz; ++z2)
                    for (int y2 = 0; y2 < by; ++y2)
                        for (int x2 = 0; x2 < bx; ++x2) {
                            int x1 = x - bx / 2 + x2, y1 = y - by / 2 + y2, z1 = z - bz / 2 + z2;
                            if (x1 >= 0 && x1 < ax && y1 >= 0 && y1 < ay && z1 >= 0 && z1 < az)
                                s += a[x1 + (long)ax * (y1 + (long)ay * z1)]
                                     * b[x2 + (long)bx * (y2 + (long)by * z2)];
                        }
                out[x + (long)ax * (y + (long)ay * z)] = s;
            }
}

#undef NW
#undef RNG
#undef SET
#undef F
