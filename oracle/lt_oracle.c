/* CPU restatement of the reference (timo-eichhorn/Lettuce) pure-gauge SU(3) hot path.
 *
 * TEST INFRASTRUCTURE ONLY -- see lt_oracle.h.  The product never links this file.
 * Plain C99, double complex arithmetic, runtime lattice extents, single thread.
 * Every routine cites the reference file:line it restates (paths relative to the
 * reference project root, LettuceGauge/...).
 */
#include "lt_oracle.h"

#include <complex.h>
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef double complex cd;
typedef struct { cd m[3][3]; } M3;

static const double PI = 3.14159265358979323846;

/* ---------------------------------------------------------------- lattice geometry */
/* site index ((t*Nx+x)*Ny+y)*Nz+z, link index site*4+mu (lattice.hpp:366-382) */
typedef struct { int n[4]; long V; } Geo;

static Geo geo(const int ext[4])
{
    Geo g;
    for (int d = 0; d < 4; ++d) g.n[d] = ext[d];
    g.V = (long)ext[0] * ext[1] * ext[2] * ext[3];
    return g;
}

static void coords(const Geo* g, long s, int c[4])
{
    c[3] = (int)(s % g->n[3]); s /= g->n[3];
    c[2] = (int)(s % g->n[2]); s /= g->n[2];
    c[1] = (int)(s % g->n[1]); s /= g->n[1];
    c[0] = (int)s;
}

static long site_of(const Geo* g, const int c[4])
{
    return (((long)c[0] * g->n[1] + c[1]) * g->n[2] + c[2]) * g->n[3] + c[3];
}

/* periodic shift by +-1 along d (lattice.hpp:249-340) */
static long move(const Geo* g, long s, int d, int dist)
{
    int c[4];
    coords(g, s, c);
    c[d] = (c[d] + dist + g->n[d]) % g->n[d];
    return site_of(g, c);
}

static M3 ld(const double* U, long site, int mu)
{
    M3 r;
    const double* p = U + 18 * (4 * site + mu);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            r.m[i][j] = p[6 * i + 2 * j] + I * p[6 * i + 2 * j + 1];
    return r;
}

static void st(double* U, long site, int mu, const M3* a)
{
    double* p = U + 18 * (4 * site + mu);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
        {
            p[6 * i + 2 * j]     = creal(a->m[i][j]);
            p[6 * i + 2 * j + 1] = cimag(a->m[i][j]);
        }
}

/* ---------------------------------------------------------------- 3x3 algebra */
static M3 zero3(void) { M3 r; memset(&r, 0, sizeof r); return r; }
static M3 id3(void) { M3 r = zero3(); r.m[0][0] = r.m[1][1] = r.m[2][2] = 1.0; return r; }

static M3 mul(M3 a, M3 b)
{
    M3 r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            r.m[i][j] = a.m[i][0] * b.m[0][j] + a.m[i][1] * b.m[1][j] + a.m[i][2] * b.m[2][j];
    return r;
}

static M3 dag(M3 a)
{
    M3 r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            r.m[i][j] = conj(a.m[j][i]);
    return r;
}

static M3 add(M3 a, M3 b)
{
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            a.m[i][j] += b.m[i][j];
    return a;
}

static M3 sub(M3 a, M3 b)
{
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            a.m[i][j] -= b.m[i][j];
    return a;
}

static M3 scl(cd s, M3 a)
{
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            a.m[i][j] *= s;
    return a;
}

static cd tr(M3 a) { return a.m[0][0] + a.m[1][1] + a.m[2][2]; }

/* SU3::Projection::Algebra: traceless anti-Hermitian part (su3.hpp:423-426) */
static M3 algebra(M3 a)
{
    M3 b = sub(a, dag(a));
    cd t = tr(b);
    M3 r = scl(0.5, b);
    for (int i = 0; i < 3; ++i) r.m[i][i] -= t / 6.0;
    return r;
}

/* SU3::Projection::TracelessHermitian (su3.hpp:445-448) */
static M3 traceless_hermitian(M3 a)
{
    M3 b = add(a, dag(a));
    cd t = tr(b);
    M3 r = scl(0.5, b);
    for (int i = 0; i < 3; ++i) r.m[i][i] -= t / 6.0;
    return r;
}

/* SU3::Projection::GramSchmidt + RestoreLastRow (su3.hpp:362-394) */
static void gram_schmidt(M3* a)
{
    double n0 = 1.0 / sqrt(creal(a->m[0][0] * conj(a->m[0][0]) + a->m[0][1] * conj(a->m[0][1])
                                 + a->m[0][2] * conj(a->m[0][2])));
    for (int n = 0; n < 3; ++n) a->m[0][n] *= n0;
    cd psi = a->m[1][0] * conj(a->m[0][0]) + a->m[1][1] * conj(a->m[0][1]) + a->m[1][2] * conj(a->m[0][2]);
    for (int n = 0; n < 3; ++n) a->m[1][n] -= psi * a->m[0][n];
    double n1 = 1.0 / sqrt(creal(a->m[1][0] * conj(a->m[1][0]) + a->m[1][1] * conj(a->m[1][1])
                                 + a->m[1][2] * conj(a->m[1][2])));
    for (int n = 0; n < 3; ++n) a->m[1][n] *= n1;
    a->m[2][0] = conj(a->m[0][1] * a->m[1][2] - a->m[0][2] * a->m[1][1]);
    a->m[2][1] = conj(a->m[0][2] * a->m[1][0] - a->m[0][0] * a->m[1][2]);
    a->m[2][2] = conj(a->m[0][0] * a->m[1][1] - a->m[0][1] * a->m[1][0]);
}

/* ---------------------------------------------------------------- Cayley-Hamilton exp */
/* ExpTaylorBounds<double> and return_xi_0 / return_xi_1 (su3_exp.hpp:38-82) */
static double xi0(double w)
{
    if (fabs(w) <= 0.05)
    {
        double w2 = w * w;
        return 1.0 - 1.0 / 6.0 * w2 * (1.0 - 1.0 / 20.0 * w2 * (1.0 - 1.0 / 42.0 * w2));
    }
    return sin(w) / w;
}

static double xi1(double w)
{
    if (fabs(w) <= 0.115)
    {
        double w2 = w * w;
        return -1.0 / 3.0 + 1.0 / 30.0 * w2 * (1.0 - 1.0 / 28.0 * w2 * (1.0 - 1.0 / 54.0 * w2));
    }
    return cos(w) / (w * w) - sin(w) / (w * w * w);
}

/* SU3::ExpConstants (su3_exp.hpp:204-283) for a traceless Hermitian Q */
typedef struct {
    M3 Q, Q2;
    double c0, c1, c0max, u, w, u2, w2, denom;
    int signflip, degenerate;
    cd emiu, e2iu, cosw, ixi0, h0, h1, h2;
} ExpC;

static ExpC exp_consts(M3 Q)
{
    ExpC e;
    e.Q = Q;
    e.Q2 = mul(Q, Q);
    double c0s = creal(tr(mul(Q, e.Q2))) / 3.0;
    e.c0 = fabs(c0s);
    e.c1 = 0.5 * creal(tr(e.Q2));
    e.c0max = 2.0 * pow(e.c1 / 3.0, 1.5);
    e.signflip = c0s < 0.0;
    double theta = acos(fmin(e.c0 / e.c0max, 1.0));
    e.u = sqrt(e.c1 / 3.0) * cos(theta / 3.0);
    e.u2 = e.u * e.u;
    e.emiu = cexp(-I * e.u);
    e.e2iu = conj(e.emiu * e.emiu);
    e.w = sqrt(e.c1) * sin(theta / 3.0);
    e.w2 = e.w * e.w;
    e.cosw = cos(e.w);
    e.ixi0 = I * xi0(e.w);
    e.degenerate = e.c0max < DBL_MIN;
    if (e.degenerate)
    {
        e.denom = 1.0; e.h0 = 1.0; e.h1 = 0.0; e.h2 = 0.0;
        return e;
    }
    double u = e.u, u2 = e.u2, w2 = e.w2;
    e.denom = 1.0 / (9.0 * u2 - w2);
    cd h0 = (u2 - w2) * e.e2iu + e.emiu * (8.0 * u2 * e.cosw + 2.0 * u * e.ixi0 * (3.0 * u2 + w2));
    cd h1 = 2.0 * u * e.e2iu - e.emiu * (2.0 * u * e.cosw - e.ixi0 * (3.0 * u2 - w2));
    cd h2 = e.e2iu - e.emiu * (e.cosw + 3.0 * u * e.ixi0);
    if (e.signflip) { h0 = conj(h0); h1 = -conj(h1); h2 = conj(h2); }
    e.h0 = h0; e.h1 = h1; e.h2 = h2;
    return e;
}

/* SU3::exp (su3_exp.hpp:419-432): exp(iQ) */
static M3 exp_from(const ExpC* e)
{
    M3 r = add(add(scl(e->h0, id3()), scl(e->h1, e->Q)), scl(e->h2, e->Q2));
    return scl(e->denom, r);
}

static M3 su3_exp(M3 Q)
{
    ExpC e = exp_consts(Q);
    return exp_from(&e);
}

void or_su3_exp(const double* q_in, double* out, int n)
{
    for (int k = 0; k < n; ++k)
    {
        M3 q, r;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                q.m[i][j] = q_in[18 * k + 6 * i + 2 * j] + I * q_in[18 * k + 6 * i + 2 * j + 1];
        r = su3_exp(q);
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
            {
                out[18 * k + 6 * i + 2 * j]     = creal(r.m[i][j]);
                out[18 * k + 6 * i + 2 * j + 1] = cimag(r.m[i][j]);
            }
    }
}

/* ---------------------------------------------------------------- staple, plaquette */
/* Rectangular<1>::StaplePlaq (rectangular_action.hpp:104-184): sum over nu != mu of
 * U_nu(x) U_mu(x+nu) U_nu(x+mu)^dag + U_nu(x-nu)^dag U_mu(x-nu) U_nu(x-nu+mu) */
static M3 staple(const Geo* g, const double* U, long s, int mu)
{
    M3 acc = zero3();
    long smu = move(g, s, mu, 1);
    for (int nu = 0; nu < 4; ++nu)
    {
        if (nu == mu) continue;
        long snu = move(g, s, nu, 1);
        long snd = move(g, s, nu, -1);
        long smu_nd = move(g, smu, nu, -1);
        M3 up = mul(mul(ld(U, s, nu), ld(U, snu, mu)), dag(ld(U, smu, nu)));
        M3 dn = mul(mul(dag(ld(U, snd, nu)), ld(U, snd, mu)), ld(U, smu_nd, nu));
        acc = add(acc, add(up, dn));
    }
    return acc;
}

/* The gauge action of staples, sweeps, HMC forces and the flow: GaugeAction::Rectangular
 * (rectangular_action.hpp:23-246) with stencil radius 1 (the plaquette staple) or 2. */
static int g_act_radius = 1;
static double g_act_cp = 1.0, g_act_cr = 0.0;

void or_set_gauge_action(int stencil_radius, double c_plaq, double c_rect)
{
    g_act_radius = stencil_radius;
    g_act_cp = c_plaq;
    g_act_cr = c_rect;
}

/* Rectangular<2>::StapleRect (rectangular_action.hpp:187-233) */
static M3 staple_rect(const Geo* g, const double* U, long s, int mu)
{
    M3 st = zero3();
    for (int off = 1; off < 4; ++off)
    {
        int nu = (mu + off) % 4;
        long nup = move(g, s, nu, 1), nupp = move(g, nup, nu, 1), mup_nup = move(g, nup, mu, 1);
        long mup = move(g, s, mu, 1);
        long nud = move(g, s, nu, -1), nudd = move(g, nud, nu, -1), mup_nudd = move(g, nudd, mu, 1);
        long mup_nud = move(g, nud, mu, 1);
        /* orthogonal to the link */
        st = add(st, add(mul(mul(mul(mul(ld(U, s, nu), ld(U, nup, nu)), ld(U, nupp, mu)), dag(ld(U, mup_nup, nu))),
                             dag(ld(U, mup, nu))),
                         mul(mul(mul(mul(dag(ld(U, nud, nu)), dag(ld(U, nudd, nu))), ld(U, nudd, mu)),
                                 ld(U, mup_nudd, nu)),
                             ld(U, mup_nud, nu))));
        /* along the link, from x */
        long mupp = move(g, mup, mu, 1), mupp_nud = move(g, mup_nud, mu, 1);
        st = add(st, mul(add(mul(mul(mul(ld(U, s, nu), ld(U, nup, mu)), ld(U, mup_nup, mu)), dag(ld(U, mupp, nu))),
                             mul(mul(mul(dag(ld(U, nud, nu)), ld(U, nud, mu)), ld(U, mup_nud, mu)), ld(U, mupp_nud, nu))),
                         dag(ld(U, mup, mu))));
        /* along the link, from x - mu */
        long mud = move(g, s, mu, -1), mud_nup = move(g, mud, nu, 1), mud_nud = move(g, mud, nu, -1);
        st = add(st, mul(dag(ld(U, mud, mu)),
                         add(mul(mul(mul(ld(U, mud, nu), ld(U, mud_nup, mu)), ld(U, nup, mu)), dag(ld(U, mup, nu))),
                             mul(mul(mul(dag(ld(U, mud_nud, nu)), ld(U, mud_nud, mu)), ld(U, nud, mu)), ld(U, mup_nud, nu)))));
    }
    return st;
}

/* Rectangular<radius>::Staple (rectangular_action.hpp:236-246) */
static M3 act_staple(const Geo* g, const double* U, long s, int mu)
{
    if (g_act_radius != 2) return staple(g, U, s, mu);
    return add(scl(g_act_cp, staple(g, U, s, mu)), scl(g_act_cr, staple_rect(g, U, s, mu)));
}

void or_staples(const int ext[4], const double* U, double* out)
{
    Geo g = geo(ext);
    for (long s = 0; s < g.V; ++s)
        for (int mu = 0; mu < 4; ++mu)
        {
            M3 a = act_staple(&g, U, s, mu);
            st(out, s, mu, &a);
        }
}

/* Plaquette (plaquette.hpp:20-24) */
static M3 plaquette(const Geo* g, const double* U, long s, int mu, int nu)
{
    return mul(mul(mul(ld(U, s, mu), ld(U, move(g, s, mu, 1), nu)), dag(ld(U, move(g, s, nu, 1), mu))),
               dag(ld(U, s, nu)));
}

/* PlaquetteSum (plaquette.hpp:26-43) */
double or_plaquette_sum(const int ext[4], const double* U)
{
    Geo g = geo(ext);
    double sum = 0.0;
    for (long s = 0; s < g.V; ++s)
        for (int nu = 1; nu < 4; ++nu)
            for (int mu = 0; mu < nu; ++mu)
                sum += creal(tr(plaquette(&g, U, s, mu, nu)));
    return sum;
}

/* Rectangular<1>::Action (rectangular_action.hpp:61-94): beta (6V - 1/3 sum ReTr P) */
double or_wilson_action(const int ext[4], const double* U, double beta)
{
    Geo g = geo(ext);
    return beta * (6.0 * (double)g.V - or_plaquette_sum(ext, U) / 3.0);
}

/* ---------------------------------------------------------------- SU(2) subgroups */
/* SU2_comp and Extract/Embed (su2.hpp:21-174) */
typedef struct { cd e11, e12; } S2;

static S2 s2_mul(S2 a, S2 b)
{
    S2 r = { a.e11 * b.e11 - a.e12 * conj(b.e12), a.e11 * b.e12 + a.e12 * conj(b.e11) };
    return r;
}
static S2 s2_adj(S2 a) { S2 r = { conj(a.e11), -a.e12 }; return r; }
static double s2_det(S2 a)
{
    return creal(a.e11) * creal(a.e11) + cimag(a.e11) * cimag(a.e11)
         + creal(a.e12) * creal(a.e12) + cimag(a.e12) * cimag(a.e12);
}
static S2 s2_scale(double s, S2 a) { a.e11 *= s; a.e12 *= s; return a; }

static const int SG[3][2] = { { 0, 1 }, { 0, 2 }, { 1, 2 } };

static S2 extract(M3 w, int g)
{
    int a = SG[g][0], b = SG[g][1];
    S2 r = { 0.5 * (w.m[a][a] + conj(w.m[b][b])), 0.5 * (w.m[a][b] - conj(w.m[b][a])) };
    return r;
}

/* Embed0x(M) * U: mixes rows a and b of U */
static M3 embed_mul(S2 m, int g, M3 u)
{
    int a = SG[g][0], b = SG[g][1];
    M3 r = u;
    for (int n = 0; n < 3; ++n)
    {
        r.m[a][n] = m.e11 * u.m[a][n] + m.e12 * u.m[b][n];
        r.m[b][n] = -conj(m.e12) * u.m[a][n] + conj(m.e11) * u.m[b][n];
    }
    return r;
}

/* OverrelaxationSubgroupKernel::OverrelaxationSU2 (overrelaxation.hpp:76-85) */
static S2 or_su2(S2 A)
{
    S2 V = s2_scale(1.0 / sqrt(s2_det(A)), A);
    return s2_adj(s2_mul(V, V));
}

/* OverrelaxationSubgroupKernel::operator() (overrelaxation.hpp:91-116) */
static void or_link(const Geo* g, double* U, long s, int mu)
{
    M3 sa = dag(act_staple(g, U, s, mu));
    M3 u = ld(U, s, mu);
    for (int sg = 0; sg < 3; ++sg)
        u = embed_mul(or_su2(extract(mul(u, sa), sg)), sg, u);
    gram_schmidt(&u);
    st(U, s, mu, &u);
}

/* Iterator::Checkerboard (iterators.hpp:65-87): for mu, for eo, all sites with
 * (t+x+y+z)&1 == eo.  Within one (mu, eo) sub-sweep the updates are independent. */
void or_overrelax_sweeps(const int ext[4], double* U, int n_sweep)
{
    Geo g = geo(ext);
    for (int sw = 0; sw < n_sweep; ++sw)
        for (int mu = 0; mu < 4; ++mu)
            for (int eo = 0; eo < 2; ++eo)
                for (long s = 0; s < g.V; ++s)
                {
                    int c[4];
                    coords(&g, s, c);
                    if (((c[0] + c[1] + c[2] + c[3]) & 1) == eo) or_link(&g, U, s, mu);
                }
}

/* ---------------------------------------------------------------- Philox4x32-10 */
void or_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3], k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r)
    {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        c1 = (uint32_t)p1;
        c3 = (uint32_t)p0;
        c0 = n0;
        c2 = n2;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* Stream layout shared with the GPU: counter words {link index, counter lo, counter hi,
 * tag<<24 | subgroup<<16 | call}, key {seed lo, seed hi}; a double is built from two words. */
enum { TAG_HEATBATH = 1, TAG_MOMENTA = 2 };

static void draw2(uint32_t link, uint64_t counter, uint32_t tagword, uint64_t seed, double d[2])
{
    uint32_t ctr[4] = { link, (uint32_t)counter, (uint32_t)(counter >> 32), tagword };
    uint32_t key[2] = { (uint32_t)seed, (uint32_t)(seed >> 32) };
    uint32_t w[4];
    or_philox4x32(ctr, key, w);
    d[0] = (double)((((uint64_t)w[0] << 32) | w[1]) >> 11) * 0x1.0p-53;
    d[1] = (double)((((uint64_t)w[2] << 32) | w[3]) >> 11) * 0x1.0p-53;
}

/* HeatbathKernel::HeatbathSU2 (heatbath.hpp:47-104); draws from the counter-based stream
 * above instead of the per-link pcg64.  Up to max_iter+1 proposals; after that the
 * reference returns the unit matrix (heatbath.hpp:73-76). */
static S2 hb_su2(S2 A, double prefactor, uint32_t link, int sg, uint64_t counter, uint64_t seed)
{
    const int max_iter = 10;
    double a_norm = 1.0 / sqrt(s2_det(A));
    S2 V = s2_scale(a_norm, A);
    double lambda_sq = 0.0;
    for (int k = 0;; ++k)
    {
        double d0[2], d1[2];
        draw2(link, counter, ((uint32_t)TAG_HEATBATH << 24) | ((uint32_t)sg << 16) | (uint32_t)(2 * k), seed, d0);
        draw2(link, counter, ((uint32_t)TAG_HEATBATH << 24) | ((uint32_t)sg << 16) | (uint32_t)(2 * k + 1), seed, d1);
        double r1 = 1.0 - d0[0], r2 = 1.0 - d0[1], r3 = 1.0 - d1[0], r0 = d1[1];
        double x1 = log(r1), x2 = cos(2.0 * PI * r2), x3 = log(r3);
        lambda_sq = -0.25 * prefactor * a_norm * (x1 + x2 * x2 * x3);
        if (k > max_iter)
        {
            S2 one = { 1.0, 0.0 };
            return one;
        }
        if (r0 * r0 + lambda_sq < 1.0) break;
    }
    double x0 = 1.0 - 2.0 * lambda_sq;
    double abs_x = sqrt(1.0 - x0 * x0);
    double da[2];
    draw2(link, counter, ((uint32_t)TAG_HEATBATH << 24) | ((uint32_t)sg << 16) | 0xFFFFu, seed, da);
    double phi = da[0];
    double cos_theta = 1.0 - 2.0 * da[1];
    double vec_norm = abs_x * sqrt(1.0 - cos_theta * cos_theta);
    S2 x = { x0 + I * (vec_norm * cos(2.0 * PI * phi)), vec_norm * sin(2.0 * PI * phi) + I * (abs_x * cos_theta) };
    return s2_mul(x, s2_adj(V));
}

/* HeatbathKernel::operator() (heatbath.hpp:110-129), prefactor 3/beta (:40) */
static void hb_link(const Geo* g, double* U, long s, int mu, double beta, uint64_t counter, uint64_t seed)
{
    M3 sa = dag(act_staple(g, U, s, mu));
    M3 u = ld(U, s, mu);
    uint32_t link = (uint32_t)(4 * s + mu);
    for (int sg = 0; sg < 3; ++sg)
        u = embed_mul(hb_su2(extract(mul(u, sa), sg), 3.0 / beta, link, sg, counter, seed), sg, u);
    gram_schmidt(&u);
    st(U, s, mu, &u);
}

void or_heatbath_sweeps(const int ext[4], double* U, double beta, int n_sweep, uint64_t seed, uint64_t counter0)
{
    Geo g = geo(ext);
    for (int sw = 0; sw < n_sweep; ++sw)
        for (int mu = 0; mu < 4; ++mu)
            for (int eo = 0; eo < 2; ++eo)
                for (long s = 0; s < g.V; ++s)
                {
                    int c[4];
                    coords(&g, s, c);
                    if (((c[0] + c[1] + c[2] + c[3]) & 1) == eo)
                        hb_link(&g, U, s, mu, beta, counter0 + (uint64_t)sw, seed);
                }
}

/* Iterator::Checkerboard4 (iterators.hpp:141-166): for mu, for sub = 0..3, the sites with
 * (t + x + y + z + x_mu) mod 4 = sub; within one sub-sweep the updates are independent. */
static int cb4_member(const Geo* g, long s, int mu, int sub)
{
    int c[4];
    coords(g, s, c);
    return (c[0] + c[1] + c[2] + c[3] + c[mu]) % 4 == sub;
}

void or_overrelax_sweeps4(const int ext[4], double* U, int n_sweep)
{
    Geo g = geo(ext);
    for (int sw = 0; sw < n_sweep; ++sw)
        for (int mu = 0; mu < 4; ++mu)
            for (int sub = 0; sub < 4; ++sub)
                for (long s = 0; s < g.V; ++s)
                    if (cb4_member(&g, s, mu, sub)) or_link(&g, U, s, mu);
}

void or_heatbath_sweeps4(const int ext[4], double* U, double beta, int n_sweep, uint64_t seed, uint64_t counter0)
{
    Geo g = geo(ext);
    for (int sw = 0; sw < n_sweep; ++sw)
        for (int mu = 0; mu < 4; ++mu)
            for (int sub = 0; sub < 4; ++sub)
                for (long s = 0; s < g.V; ++s)
                    if (cb4_member(&g, s, mu, sub)) hb_link(&g, U, s, mu, beta, counter0 + (uint64_t)sw, seed);
}

/* ---------------------------------------------------------------- gradient flow */
/* Z = c_old * Z + c_new * Algebra(st U^dag) (gradient_flow.hpp:298-332) */
static void flow_z(const Geo* g, const double* U, double* Z, double c_old, double c_new)
{
    for (long s = 0; s < g->V; ++s)
        for (int mu = 0; mu < 4; ++mu)
        {
            M3 a = algebra(mul(act_staple(g, U, s, mu), dag(ld(U, s, mu))));
            M3 z = c_old == 0.0 ? scl(c_new, a) : add(scl(c_old, ld(Z, s, mu)), scl(c_new, a));
            st(Z, s, mu, &z);
        }
}

/* U = exp(c Z) U, then Gram-Schmidt (gradient_flow.hpp:265-282); exp(cZ) = SU3::exp(-i c Z) */
static void flow_update(const Geo* g, double* U, const double* Z, double c)
{
    for (long s = 0; s < g->V; ++s)
        for (int mu = 0; mu < 4; ++mu)
        {
            M3 u = mul(su3_exp(scl(-I * c, ld(Z, s, mu))), ld(U, s, mu));
            gram_schmidt(&u);
            st(U, s, mu, &u);
        }
}

/* Integrators::GradientFlow::RK3 (gradient_flow.hpp:120-168) */
void or_flow_rk3(const int ext[4], const double* in, double* out, double eps, int n_step)
{
    Geo g = geo(ext);
    size_t n = (size_t)g.V * 4 * 18;
    double* Z = (double*)calloc(n, sizeof(double));
    if (out != in) memcpy(out, in, n * sizeof(double));
    for (int k = 0; k < n_step; ++k)
    {
        flow_z(&g, out, Z, 0.0, eps);
        flow_update(&g, out, Z, 0.25);
        flow_z(&g, out, Z, -17.0 / 36.0, 8.0 / 9.0 * eps);
        flow_update(&g, out, Z, 1.0);
        flow_z(&g, out, Z, -1.0, 3.0 / 4.0 * eps);
        flow_update(&g, out, Z, 1.0);
    }
    free(Z);
}

/* Integrators::GradientFlow::Euler, RK2, RK3, RK3W7 (gradient_flow.hpp:31-56, :88-113,
 * :114-140, :142-168): the same Z / field update steps with the integrators' coefficients.
 * integrator: 0 Euler, 1 RK2, 2 RK3, 3 RK3W7 */
void or_flow(const int ext[4], const double* in, double* out, double eps, int n_step, int integrator)
{
    if (integrator == 2)
    {
        or_flow_rk3(ext, in, out, eps, n_step);
        return;
    }
    Geo g = geo(ext);
    size_t n = (size_t)g.V * 4 * 18;
    double* Z = (double*)calloc(n, sizeof(double));
    if (out != in) memcpy(out, in, n * sizeof(double));
    for (int k = 0; k < n_step; ++k)
    {
        if (integrator == 0)
        {
            flow_z(&g, out, Z, 0.0, eps);
            flow_update(&g, out, Z, 1.0);
        }
        else if (integrator == 1)
        {
            flow_z(&g, out, Z, 0.0, eps);
            flow_update(&g, out, Z, 0.5);
            flow_z(&g, out, Z, -0.5, eps);
            flow_update(&g, out, Z, 1.0);
        }
        else
        {
            flow_z(&g, out, Z, 0.0, eps);
            flow_update(&g, out, Z, 1.0 / 3.0);
            flow_z(&g, out, Z, -25.0 / 48.0, 15.0 / 16.0 * eps);
            flow_update(&g, out, Z, 1.0);
            flow_z(&g, out, Z, -17.0 / 25.0, 8.0 / 15.0 * eps);
            flow_update(&g, out, Z, 1.0);
        }
    }
    free(Z);
}

/* ---------------------------------------------------------------- Zeuthen flow */
/* The Zeuthen flow (Ramos and Sint, Eur. Phys. J. C 76 (2016) 15, arXiv:1508.05552; not in the
 * reference, parity unpinned): the force is the Luescher-Weisz action's, X = Algebra(st_LW U^dag)
 * (c_plaq = 5/3, c_rect = -1/12), acted on by 1 + (1/12) nabla*_mu nabla_mu with the adjoint
 * covariant differences along the link direction:
 *   nabla_mu w(x)  = U_mu(x) w(x+mu) U_mu(x)^dag - w(x)
 *   nabla*_mu w(x) = w(x) - U_mu(x-mu)^dag w(x-mu) U_mu(x-mu)
 * Z = c_old Z + c_new Algebra(X + nabla*_mu nabla_mu X / 12), then the integrator's update. */
static void flow_z_zeuthen(const Geo* g, const double* U, double* Z, double* X, double c_old, double c_new)
{
    const int r0 = g_act_radius;
    const double cp0 = g_act_cp, cr0 = g_act_cr;
    long s;
    int mu;
    or_set_gauge_action(2, 5.0 / 3.0, -1.0 / 12.0);
    for (s = 0; s < g->V; ++s)
        for (mu = 0; mu < 4; ++mu)
        {
            M3 x = algebra(mul(act_staple(g, U, s, mu), dag(ld(U, s, mu))));
            st(X, s, mu, &x);
        }
    or_set_gauge_action(r0, cp0, cr0);
    for (s = 0; s < g->V; ++s)
        for (mu = 0; mu < 4; ++mu)
        {
            long sp = move(g, s, mu, 1), sm = move(g, s, mu, -1);
            M3 u = ld(U, s, mu), um = ld(U, sm, mu), x = ld(X, s, mu);
            /* nabla w at x and at x - mu, then the backward difference of the two */
            M3 dx = add(mul(mul(u, ld(X, sp, mu)), dag(u)), scl(-1.0, x));
            M3 dxm = add(mul(mul(um, x), dag(um)), scl(-1.0, ld(X, sm, mu)));
            M3 lap = add(dx, scl(-1.0, mul(mul(dag(um), dxm), um)));
            M3 a = algebra(add(x, scl(1.0 / 12.0, lap)));
            M3 z = c_old == 0.0 ? scl(c_new, a) : add(scl(c_old, ld(Z, s, mu)), scl(c_new, a));
            st(Z, s, mu, &z);
        }
}

/* The Zeuthen flow integrated with the stages of Integrators::GradientFlow (0 Euler, 1 RK2,
 * 2 RK3, 3 RK3W7; gradient_flow.hpp:31-168) */
void or_flow_zeuthen(const int ext[4], const double* in, double* out, double eps, int n_step, int integrator)
{
    static const double stages[4][3][3] = {
        { { 0.0, 1.0, 1.0 } },
        { { 0.0, 1.0, 0.5 }, { -0.5, 1.0, 1.0 } },
        { { 0.0, 1.0, 0.25 }, { -17.0 / 36.0, 8.0 / 9.0, 1.0 }, { -1.0, 3.0 / 4.0, 1.0 } },
        { { 0.0, 1.0, 1.0 / 3.0 }, { -25.0 / 48.0, 15.0 / 16.0, 1.0 }, { -17.0 / 25.0, 8.0 / 15.0, 1.0 } } };
    static const int n_stage[4] = { 1, 2, 3, 3 };
    Geo g = geo(ext);
    size_t n = (size_t)g.V * 4 * 18;
    double* Z = (double*)calloc(n, sizeof(double));
    double* X = (double*)calloc(n, sizeof(double));
    int k, j;
    if (out != in) memcpy(out, in, n * sizeof(double));
    for (k = 0; k < n_step; ++k)
        for (j = 0; j < n_stage[integrator]; ++j)
        {
            flow_z_zeuthen(&g, out, Z, X, stages[integrator][j][0], stages[integrator][j][1] * eps);
            flow_update(&g, out, Z, stages[integrator][j][2]);
        }
    free(Z);
    free(X);
}

/* ---------------------------------------------------------------- stout smearing */
/* StoutSmearing4D (stout_smearing.hpp:29-57) */
static void stout_step(const Geo* g, const double* in, double* out, double rho)
{
    for (long s = 0; s < g->V; ++s)
        for (int mu = 0; mu < 4; ++mu)
        {
            M3 u = ld(in, s, mu);
            M3 C = algebra(mul(staple(g, in, s, mu), dag(u)));
            M3 r = mul(su3_exp(scl(-I * rho, C)), u);
            gram_schmidt(&r);
            st(out, s, mu, &r);
        }
}

void or_stout(const int ext[4], const double* in, double* out, double rho, int n)
{
    Geo g = geo(ext);
    size_t sz = (size_t)g.V * 4 * 18 * sizeof(double);
    double* a = (double*)malloc(sz);
    double* b = (double*)malloc(sz);
    memcpy(a, in, sz);
    for (int k = 0; k < n; ++k)
    {
        stout_step(&g, a, b, rho);
        double* t = a; a = b; b = t;
    }
    memcpy(out, a, sz);
    free(a);
    free(b);
}

/* ---------------------------------------------------------------- clover */
/* Four-leaf clover C_mu,nu = PlaquetteI + II + III + IV (plaquette.hpp:82-114,
 * clover.hpp:40-52) */
static M3 clover(const Geo* g, const double* U, long s, int mu, int nu)
{
    long smd = move(g, s, mu, -1), snd = move(g, s, nu, -1);
    long smd_nd = move(g, smd, nu, -1);
    M3 p1 = plaquette(g, U, s, mu, nu);
    M3 p2 = mul(mul(mul(ld(U, s, nu), dag(ld(U, move(g, smd, nu, 1), mu))), dag(ld(U, smd, nu))), ld(U, smd, mu));
    M3 p3 = mul(mul(mul(dag(ld(U, smd, mu)), dag(ld(U, smd_nd, nu))), ld(U, smd_nd, mu)), ld(U, snd, nu));
    M3 p4 = mul(mul(mul(dag(ld(U, snd, nu)), ld(U, snd, mu)), ld(U, move(g, snd, mu, 1), nu)), dag(ld(U, s, mu)));
    return add(add(p1, p2), add(p3, p4));
}

/* TopChargeClover (topological_charge.hpp:97-200): F = C - C^dag, no trace subtraction */
double or_topcharge_clover(const int ext[4], const double* U)
{
    Geo g = geo(ext);
    double q = 0.0;
    for (long s = 0; s < g.V; ++s)
    {
        M3 F[4][4];
        for (int mu = 0; mu < 4; ++mu)
            for (int nu = mu + 1; nu < 4; ++nu)
            {
                M3 c = clover(&g, U, s, mu, nu);
                F[mu][nu] = sub(c, dag(c));
            }
        q += creal(tr(sub(add(mul(F[0][1], F[2][3]), mul(F[0][3], F[1][2])), mul(F[0][2], F[1][3]))));
    }
    return -1.0 / (64.0 * 4.0 * PI * PI) * q;
}

/* EnergyDensity::Clover on the traceless clover field strength
 * (field_strength_tensor.hpp:28-66, :107-134, :154-175): F = Traceless(-i/4 * AH(C)) */
double or_energy_clover(const int ext[4], const double* U)
{
    Geo g = geo(ext);
    double e = 0.0;
    for (long s = 0; s < g.V; ++s)
        for (int mu = 0; mu < 4; ++mu)
            for (int nu = mu + 1; nu < 4; ++nu)
            {
                M3 c = clover(&g, U, s, mu, nu);
                M3 f = scl(-I / 4.0, scl(0.5, sub(c, dag(c))));
                cd t = tr(f) / 3.0;
                for (int i = 0; i < 3; ++i) f.m[i][i] -= t;
                e += creal(tr(mul(f, f)));
            }
    return e / (double)g.V;
}

/* ---------------------------------------------------------------- HMC pieces */
/* gauge force beta/6 Algebra(st U^dag) (hmc_gauge.hpp:450-464) */
void or_gauge_force(const int ext[4], const double* U, double beta, double* out)
{
    Geo g = geo(ext);
    for (long s = 0; s < g.V; ++s)
        for (int mu = 0; mu < 4; ++mu)
        {
            M3 f = scl(beta / 6.0, algebra(mul(act_staple(&g, U, s, mu), dag(ld(U, s, mu)))));
            st(out, s, mu, &f);
        }
}

/* -sum ReTr(P^2) (hmc_gauge.hpp:525-541) */
double or_kinetic(const int ext[4], const double* P)
{
    Geo g = geo(ext);
    double k = 0.0;
    for (long s = 0; s < g.V; ++s)
        for (int mu = 0; mu < 4; ++mu)
        {
            M3 p = ld(P, s, mu);
            k -= creal(tr(mul(p, p)));
        }
    return k;
}

/* RandomMomentum (hmc_gauge.hpp:400-428) from the counter-based Gaussian stream:
 * call j = 0..3 gives two uniforms (u1, u2) -> Box-Muller pair (phi_{2j+1}, phi_{2j+2}). */
void or_random_momenta(const int ext[4], double* P, uint64_t seed, uint64_t counter)
{
    Geo g = geo(ext);
    const double s3 = sqrt(3.0);
    for (long s = 0; s < g.V; ++s)
        for (int mu = 0; mu < 4; ++mu)
        {
            double phi[8];
            uint32_t link = (uint32_t)(4 * s + mu);
            for (int j = 0; j < 4; ++j)
            {
                double d[2];
                draw2(link, counter, ((uint32_t)TAG_MOMENTA << 24) | (uint32_t)j, seed, d);
                double r = sqrt(-2.0 * log(1.0 - d[0]));
                phi[2 * j]     = r * cos(2.0 * PI * d[1]);
                phi[2 * j + 1] = r * sin(2.0 * PI * d[1]);
            }
            M3 a;
            a.m[0][0] = I * (phi[2] + phi[7] / s3);
            a.m[0][1] = phi[1] + I * phi[0];
            a.m[0][2] = phi[4] + I * phi[3];
            a.m[1][0] = -phi[1] + I * phi[0];
            a.m[1][1] = I * (-phi[2] + phi[7] / s3);
            a.m[1][2] = phi[6] + I * phi[5];
            a.m[2][0] = -phi[4] + I * phi[3];
            a.m[2][1] = -phi[6] + I * phi[5];
            a.m[2][2] = I * (-2.0 * phi[7] / s3);
            a = scl(0.5, a);
            st(P, s, mu, &a);
        }
}

static void hmc_update_momenta(const Geo* g, const double* U, double* P, double beta, double eps,
                               const double* extra)
{
    for (long s = 0; s < g->V; ++s)
        for (int mu = 0; mu < 4; ++mu)
        {
            M3 f = scl(beta / 6.0, algebra(mul(act_staple(g, U, s, mu), dag(ld(U, s, mu)))));
            if (extra) f = add(f, ld(extra, s, mu));
            M3 p = add(ld(P, s, mu), scl(eps, f));
            st(P, s, mu, &p);
        }
}

/* HMCKernel::UpdateFields (hmc_gauge.hpp:505-523) */
static void hmc_update_fields(const Geo* g, double* U, const double* P, double eps)
{
    for (long s = 0; s < g->V; ++s)
        for (int mu = 0; mu < 4; ++mu)
        {
            M3 u = mul(su3_exp(scl(-I * eps, ld(P, s, mu))), ld(U, s, mu));
            gram_schmidt(&u);
            st(U, s, mu, &u);
        }
}

/* Integrators::HMC::OMF_2 (hmc_gauge.hpp:155-190) with merged kicks */
void or_omf2(const int ext[4], double* U, double* P, double beta, double tau, int n_step,
             double* h_old, double* h_new)
{
    Geo g = geo(ext);
    const double lam = 0.1931833275037836;
    double eps = tau / n_step, a = lam * eps, b = 0.5 * eps, c = (1.0 - 2.0 * lam) * eps;
    *h_old = or_wilson_action(ext, U, beta) + or_kinetic(ext, P);
    hmc_update_momenta(&g, U, P, beta, a, NULL);
    hmc_update_fields(&g, U, P, b);
    hmc_update_momenta(&g, U, P, beta, c, NULL);
    hmc_update_fields(&g, U, P, b);
    for (int k = 0; k < n_step - 1; ++k)
    {
        hmc_update_momenta(&g, U, P, beta, 2.0 * a, NULL);
        hmc_update_fields(&g, U, P, b);
        hmc_update_momenta(&g, U, P, beta, c, NULL);
        hmc_update_fields(&g, U, P, b);
    }
    hmc_update_momenta(&g, U, P, beta, a, NULL);
    *h_new = or_wilson_action(ext, U, beta) + or_kinetic(ext, P);
}

/* ---------------------------------------------------------------- clover derivative */
/* CloverDerivativeComponent (clover.hpp:238-276) with R = C_rho,sigma - C_sigma,rho */
static M3 clover_R(const M3* C, long s, int rho, int sigma)
{
    /* C holds the six C_mu<nu per site; C_nu,mu = C_mu,nu^dag (clover.hpp:94-152) */
    static const int plane[4][4] = { { -1, 0, 1, 2 }, { 0, -1, 3, 4 }, { 1, 3, -1, 5 }, { 2, 4, 5, -1 } };
    M3 c = C[6 * s + plane[rho][sigma]];
    if (rho < sigma) return sub(c, dag(c));
    return sub(dag(c), c);
}

static M3 clover_deriv_component(const Geo* g, const double* U, const M3* C, long s, int mu, int nu, int rho, int sigma)
{
    long smu = move(g, s, mu, 1), snu = move(g, s, nu, 1), snd = move(g, s, nu, -1);
    long smu_nu = move(g, smu, nu, 1), smu_nd = move(g, smu, nu, -1);
    M3 R_s = clover_R(C, s, rho, sigma), R_nup = clover_R(C, snu, rho, sigma);
    M3 R_mupnup = clover_R(C, smu_nu, rho, sigma), R_mup = clover_R(C, smu, rho, sigma);
    M3 R_nud = clover_R(C, snd, rho, sigma), R_mupnud = clover_R(C, smu_nd, rho, sigma);
    M3 t1 = mul(ld(U, smu, nu), dag(ld(U, snu, mu)));
    M3 t2 = mul(dag(ld(U, snu, mu)), dag(ld(U, s, nu)));
    M3 t3 = mul(dag(ld(U, smu_nd, nu)), dag(ld(U, snd, mu)));
    M3 t4 = mul(dag(ld(U, snd, mu)), ld(U, snd, nu));
    M3 r = mul(t1, add(mul(dag(ld(U, s, nu)), R_s), mul(R_nup, dag(ld(U, s, nu)))));
    r = add(r, mul(add(mul(ld(U, smu, nu), R_mupnup), mul(R_mup, ld(U, smu, nu))), t2));
    r = sub(r, mul(t3, add(mul(ld(U, snd, nu), R_s), mul(R_nud, ld(U, snd, nu)))));
    r = sub(r, mul(add(mul(dag(ld(U, smu_nd, nu)), R_mupnud), mul(R_mup, dag(ld(U, smu_nd, nu)))), t4));
    return r;
}

static M3* clover_field(const Geo* g, const double* U)
{
    M3* C = (M3*)malloc(sizeof(M3) * 6 * (size_t)g->V);
    for (long s = 0; s < g->V; ++s)
    {
        int k = 0;
        for (int mu = 0; mu < 4; ++mu)
            for (int nu = mu + 1; nu < 4; ++nu)
                C[6 * s + k++] = clover(g, U, s, mu, nu);
    }
    return C;
}

/* CloverDerivative (clover.hpp:279-321) */
static M3 clover_derivative(const Geo* g, const double* U, const M3* C, long s, int mu)
{
    /* the three epsilon terms (nu, rho, sigma) with signs, per direction mu */
    static const int terms[4][3][4] = {
        { { +1, 1, 2, 3 }, { -1, 2, 1, 3 }, { +1, 3, 1, 2 } },
        { { -1, 0, 2, 3 }, { +1, 2, 0, 3 }, { -1, 3, 0, 2 } },
        { { +1, 0, 1, 3 }, { -1, 1, 0, 3 }, { +1, 3, 0, 1 } },
        { { -1, 0, 1, 2 }, { +1, 1, 0, 2 }, { -1, 2, 0, 1 } } };
    M3 d = zero3();
    for (int k = 0; k < 3; ++k)
    {
        M3 c = clover_deriv_component(g, U, C, s, mu, terms[mu][k][1], terms[mu][k][2], terms[mu][k][3]);
        d = terms[mu][k][0] > 0 ? add(d, c) : sub(d, c);
    }
    d = mul(ld(U, s, mu), d);
    return scl(-2.0 / (512.0 * PI * PI), algebra(d));
}

void or_clover_derivative(const int ext[4], const double* U, double* out)
{
    Geo g = geo(ext);
    M3* C = clover_field(&g, U);
    for (long s = 0; s < g.V; ++s)
        for (int mu = 0; mu < 4; ++mu)
        {
            M3 d = clover_derivative(&g, U, C, s, mu);
            st(out, s, mu, &d);
        }
    free(C);
}

/* ---------------------------------------------------------------- stout force recursion */
/* ExpDerivativeConstants r, b coefficients and B_1, B_2 (su3_exp.hpp:121-201, :389-415) */
typedef struct { cd f1, f2; M3 B1, B2; } ExpD;

static ExpD exp_deriv(const ExpC* e)
{
    ExpD r;
    double u = e->u, u2 = e->u2, w2 = e->w2;
    cd x0 = xi0(e->w), x1 = xi1(e->w);
    cd f0 = e->denom * e->h0, f1 = e->denom * e->h1, f2 = e->denom * e->h2;
    cd emiu = e->emiu, e2iu = e->e2iu, cosw = e->cosw, ix0 = e->ixi0;
    cd r10 = 2.0 * (u + I * (u2 - w2)) * e2iu
           + 2.0 * emiu * (4.0 * u * (2.0 - I * u) * cosw + ix0 * (9.0 * u2 + w2 - I * u * (3.0 * u2 + w2)));
    cd r11 = 2.0 * (1.0 + 2.0 * I * u) * e2iu + emiu * (-2.0 * (1.0 - I * u) * cosw + ix0 * (6.0 * u + I * (w2 - 3.0 * u2)));
    cd r12 = 2.0 * I * e2iu + I * emiu * (cosw - 3.0 * (1.0 - I * u) * x0);
    cd r20 = -2.0 * e2iu + 2.0 * I * u * emiu * (cosw + (1.0 + 4.0 * I * u) * x0 + 3.0 * u2 * x1);
    cd r21 = -I * emiu * (cosw + (1.0 + 2.0 * I * u) * x0 - 3.0 * u2 * x1);
    cd r22 = emiu * (x0 - 3.0 * I * u * x1);
    cd b10, b11, b12, b20, b21, b22;
    if (e->c0max < DBL_MIN)
    {
        b10 = b11 = b12 = b20 = b21 = b22 = 0.0;
    }
    else
    {
        double bd = 9.0 * u2 - w2;
        bd *= 2.0 * bd;
        bd = 1.0 / bd;
        double k1 = 3.0 * u2 - w2, k2 = 2.0 * (15.0 * u2 + w2);
        if (e->signflip)
        {
            b10 =  bd * conj(2.0 * u * r10 + k1 * r20 - k2 * conj(f0));
            b11 = -bd * conj(2.0 * u * r11 + k1 * r21 - k2 * -conj(f1));
            b12 =  bd * conj(2.0 * u * r12 + k1 * r22 - k2 * conj(f2));
            b20 = -bd * conj(r10 - 3.0 * u * r20 - 24.0 * u * conj(f0));
            b21 =  bd * conj(r11 - 3.0 * u * r21 - 24.0 * u * -conj(f1));
            b22 = -bd * conj(r12 - 3.0 * u * r22 - 24.0 * u * conj(f2));
        }
        else
        {
            b10 = bd * (2.0 * u * r10 + k1 * r20 - k2 * f0);
            b11 = bd * (2.0 * u * r11 + k1 * r21 - k2 * f1);
            b12 = bd * (2.0 * u * r12 + k1 * r22 - k2 * f2);
            b20 = bd * (r10 - 3.0 * u * r20 - 24.0 * u * f0);
            b21 = bd * (r11 - 3.0 * u * r21 - 24.0 * u * f1);
            b22 = bd * (r12 - 3.0 * u * r22 - 24.0 * u * f2);
        }
    }
    r.f1 = f1;
    r.f2 = f2;
    r.B1 = add(add(scl(b10, id3()), scl(b11, e->Q)), scl(b12, e->Q2));
    r.B2 = add(add(scl(b20, id3()), scl(b21, e->Q)), scl(b22, e->Q2));
    return r;
}

/* StoutForceRecursion (stout_smearing.hpp:152-234) with CalculateLambda (:122-150).
 * U = level k-1, Up = level k; Sigma (level k force, algebra valued) -> level k-1 force. */
static void stout_force_recursion(const Geo* g, const double* U, const double* Up, double* Sigma, double rho)
{
    size_t nl = (size_t)g->V * 4;
    M3* Lam = (M3*)malloc(sizeof(M3) * nl);
    M3* Sp = (M3*)malloc(sizeof(M3) * nl);
    ExpC* E = (ExpC*)malloc(sizeof(ExpC) * nl);
    for (long s = 0; s < g->V; ++s)
        for (int mu = 0; mu < 4; ++mu)
        {
            size_t l = 4 * (size_t)s + mu;
            Sp[l] = mul(dag(ld(Up, s, mu)), ld(Sigma, s, mu));
            M3 u = ld(U, s, mu);
            M3 C = algebra(mul(staple(g, U, s, mu), dag(u)));
            E[l] = exp_consts(scl(-I * rho, C));
            ExpD d = exp_deriv(&E[l]);
            M3 tmp = mul(u, Sp[l]);
            M3 lam = add(add(scl(tr(mul(d.B1, tmp)), E[l].Q), scl(tr(mul(d.B2, tmp)), E[l].Q2)),
                         add(scl(d.f1, tmp), scl(d.f2, add(mul(E[l].Q, tmp), mul(tmp, E[l].Q)))));
            Lam[l] = traceless_hermitian(lam);
        }
#define LAM(site, dir) Lam[4 * (size_t)(site) + (dir)]
    for (long s = 0; s < g->V; ++s)
        for (int mu = 0; mu < 4; ++mu)
        {
            size_t l = 4 * (size_t)s + mu;
            M3 fs = zero3();
            for (int nu = 0; nu < 4; ++nu)
            {
                if (nu == mu) continue;
                long smu = move(g, s, mu, 1), snu = move(g, s, nu, 1), snd = move(g, s, nu, -1);
                long smu_nd = move(g, smu, nu, -1);
                M3 t1 = mul(ld(U, smu, nu), dag(ld(U, snu, mu)));
                M3 t2 = mul(dag(ld(U, snd, mu)), sub(LAM(snd, mu), LAM(snd, nu)));
                M3 a = mul(t1, add(mul(dag(ld(U, s, nu)), LAM(s, nu)), mul(LAM(snu, mu), dag(ld(U, s, nu)))));
                M3 b = mul(mul(dag(ld(U, smu_nd, nu)), add(t2, mul(LAM(smu_nd, nu), dag(ld(U, snd, mu))))), ld(U, snd, nu));
                M3 c = mul(mul(LAM(smu, nu), t1), dag(ld(U, s, nu)));
                fs = add(fs, sub(add(a, b), c));
            }
            M3 Cadj = scl(rho, dag(staple(g, U, s, mu)));
            M3 inner = add(mul(Sp[l], exp_from(&E[l])), scl(I, mul(Cadj, LAM(s, mu))));
            inner = sub(inner, scl(I * rho, fs));
            M3 out = algebra(mul(ld(U, s, mu), inner));
            st(Sigma, s, mu, &out);
        }
#undef LAM
    free(Lam);
    free(Sp);
    free(E);
}

/* HMCMetaDKernel::CalculateTopologicalForce (hmc_metadynamics.hpp:374-436) for n_stout
 * levels: forward stout (storing each level), clover, dV/dQ * clover derivative on the
 * most smeared field, then the recursion back to the thin links.  Returns Q_smeared. */
double or_metad_force(const int ext[4], const double* U, double rho, int n_stout, double dvdq, double* out)
{
    Geo g = geo(ext);
    size_t n = (size_t)g.V * 4 * 18;
    double** lv = (double**)malloc(sizeof(double*) * (size_t)(n_stout + 1));
    for (int k = 0; k <= n_stout; ++k) lv[k] = (double*)malloc(n * sizeof(double));
    memcpy(lv[0], U, n * sizeof(double));
    for (int k = 0; k < n_stout; ++k) stout_step(&g, lv[k], lv[k + 1], rho);
    double q = or_topcharge_clover(ext, lv[n_stout]);
    M3* C = clover_field(&g, lv[n_stout]);
    for (long s = 0; s < g.V; ++s)
        for (int mu = 0; mu < 4; ++mu)
        {
            M3 d = scl(dvdq, clover_derivative(&g, lv[n_stout], C, s, mu));
            st(out, s, mu, &d);
        }
    free(C);
    for (int k = n_stout; k > 0; --k) stout_force_recursion(&g, lv[k - 1], lv[k], out, rho);
    for (int k = 0; k <= n_stout; ++k) free(lv[k]);
    free(lv);
    return q;
}

double or_metad_charge(const int ext[4], const double* U, double rho, int n_stout)
{
    Geo g = geo(ext);
    size_t n = (size_t)g.V * 4 * 18;
    double* s = (double*)malloc(n * sizeof(double));
    or_stout(ext, U, s, rho, n_stout);
    double q = or_topcharge_clover(ext, s);
    free(s);
    return q;
}

/* ---------------------------------------------------------------- MD integrators */
/* The integrators of updates/hmc_gauge.hpp:19-377 and updates/hmc_metadynamics.hpp:26-238,
 * driven through the five momentum/field updates below.  With metad != 0 the bias is linear,
 * V(Q) = slope * Q, and its force slope * dQ_stout/dU is evaluated at the current links at
 * every full or Metadynamics momentum update. */
typedef struct
{
    const int* ext;
    Geo g;
    double *U, *P, *F, beta, rho, slope;
    int metad, n_stout;
} MdState;

/* UpdateMomenta (hmc_gauge.hpp:450-464; hmc_metadynamics.hpp:441-459 under MetaD) */
static void md_kick(MdState* s, double eps)
{
    if (s->metad) or_metad_force(s->ext, s->U, s->rho, s->n_stout, s->slope, s->F);
    hmc_update_momenta(&s->g, s->U, s->P, s->beta, eps, s->metad ? s->F : NULL);
}

/* UpdateGaugeMomenta (hmc_metadynamics.hpp:464-476) */
static void md_kick_gauge(MdState* s, double eps) { hmc_update_momenta(&s->g, s->U, s->P, s->beta, eps, NULL); }

/* UpdateMetadynamicsMomenta (hmc_metadynamics.hpp:478-491) with the force at the current links */
static void md_kick_metad(MdState* s, double eps)
{
    or_metad_force(s->ext, s->U, s->rho, s->n_stout, s->slope, s->F);
    for (long x = 0; x < s->g.V; ++x)
        for (int mu = 0; mu < 4; ++mu)
        {
            M3 p = add(ld(s->P, x, mu), scl(eps, ld(s->F, x, mu)));
            st(s->P, x, mu, &p);
        }
}

/* UpdateMomentaFriction (hmc_gauge.hpp:469-503) */
static void md_friction(MdState* s, double eps, double fric, int without_kick)
{
    const double e = exp(-fric * eps);
    for (long x = 0; x < s->g.V; ++x)
        for (int mu = 0; mu < 4; ++mu)
        {
            M3 f = scl(eps * s->beta / 6.0, algebra(mul(act_staple(&s->g, s->U, x, mu), dag(ld(s->U, x, mu)))));
            M3 p = without_kick ? add(scl(e, ld(s->P, x, mu)), f) : scl(e, add(ld(s->P, x, mu), f));
            st(s->P, x, mu, &p);
        }
}

static void md_drift(MdState* s, double eps) { hmc_update_fields(&s->g, s->U, s->P, eps); }

static const double OMF2_L = 0.1931833275037836;
static const double OMF4_A = 0.08398315262876693, OMF4_B = 0.2539785108410595, OMF4_G = 0.6822365335719091,
                    OMF4_D = -0.03230286765269967;

/* the middle of one OMF4 step (everything between its first and last momentum update) at
 * step size e, kicks by UpdateGaugeMomenta (gauge_only) or UpdateMomenta */
static void md_omf4_middle(MdState* s, double e, int gauge_only)
{
    const double mu = 0.5 - OMF4_G - OMF4_A, nu = 1.0 - 2.0 * OMF4_D - 2.0 * OMF4_B;
    void (*k)(MdState*, double) = gauge_only ? md_kick_gauge : md_kick;
    md_drift(s, OMF4_B * e);
    k(s, OMF4_G * e);
    md_drift(s, OMF4_D * e);
    k(s, mu * e);
    md_drift(s, nu * e);
    k(s, mu * e);
    md_drift(s, OMF4_D * e);
    k(s, OMF4_G * e);
    md_drift(s, OMF4_B * e);
}

static void md_friction_step(MdState* s, int omf4, double e, double* fric, int flip_mid)
{
    if (!omf4)
    {
        md_friction(s, 0.5 * e, *fric, 1);
        md_drift(s, e);
        if (flip_mid) *fric = -*fric;
        md_friction(s, 0.5 * e, *fric, 0);
        return;
    }
    const double mu = 0.5 - OMF4_G - OMF4_A, nu = 1.0 - 2.0 * OMF4_D - 2.0 * OMF4_B;
    md_friction(s, OMF4_A * e, *fric, 1);
    md_drift(s, OMF4_B * e);
    md_friction(s, OMF4_G * e, *fric, 1);
    md_drift(s, OMF4_D * e);
    md_friction(s, mu * e, *fric, 1);
    md_drift(s, nu * e);
    if (flip_mid) *fric = -*fric;
    md_friction(s, mu * e, *fric, 0);
    md_drift(s, OMF4_D * e);
    md_friction(s, OMF4_G * e, *fric, 0);
    md_drift(s, OMF4_B * e);
    md_friction(s, OMF4_A * e, *fric, 0);
}

/* Action(U) of the current gauge action (rectangular_action.hpp:61-94) */
static double act_action(const int ext[4], const double* U, double beta)
{
    if (g_act_radius == 2) return or_rect_action(ext, U, beta, g_act_cp, g_act_cr);
    Geo g = geo(ext);
    return beta * g_act_cp * (6.0 * (double)g.V - or_plaquette_sum(ext, U) / 3.0);
}

static double md_energy(MdState* s)
{
    double h = act_action(s->ext, s->U, s->beta) + or_kinetic(s->ext, s->P);
    if (s->metad) h += s->slope * or_metad_charge(s->ext, s->U, s->rho, s->n_stout);
    return h;
}

void or_md_integrate(const int ext[4], double* U, double* P, double beta, double tau, int n, int integrator,
                     int metad, double rho, int n_stout, double slope, double* h_old, double* h_new)
{
    MdState s;
    s.ext = ext;
    s.g = geo(ext);
    s.U = U;
    s.P = P;
    s.F = (double*)malloc(sizeof(double) * (size_t)s.g.V * 72);
    s.beta = beta;
    s.rho = rho;
    s.slope = slope;
    s.metad = metad;
    s.n_stout = n_stout;
    *h_old = md_energy(&s);
    const double e = n > 0 ? tau / n : 0.0;
    const double l2 = OMF2_L, a4 = OMF4_A;
    if (n > 0) switch (integrator)
    {
    case 0:   /* Leapfrog_slow (hmc_gauge.hpp:21-44) */
        for (int k = 0; k < n; ++k) { md_kick(&s, 0.5 * e); md_drift(&s, e); md_kick(&s, 0.5 * e); }
        break;
    case 1:   /* Leapfrog (:47-70) */
        md_kick(&s, 0.5 * e);
        for (int k = 0; k < n - 1; ++k) { md_drift(&s, e); md_kick(&s, e); }
        md_drift(&s, e);
        md_kick(&s, 0.5 * e);
        break;
    case 2:   /* OMF_2_slow (:121-151) */
        for (int k = 0; k < n; ++k)
        {
            md_kick(&s, l2 * e); md_drift(&s, 0.5 * e); md_kick(&s, (1.0 - 2.0 * l2) * e);
            md_drift(&s, 0.5 * e); md_kick(&s, l2 * e);
        }
        break;
    case 3:   /* OMF_2 (:155-190) */
        md_kick(&s, l2 * e); md_drift(&s, 0.5 * e); md_kick(&s, (1.0 - 2.0 * l2) * e); md_drift(&s, 0.5 * e);
        for (int k = 0; k < n - 1; ++k)
        {
            md_kick(&s, 2.0 * l2 * e); md_drift(&s, 0.5 * e); md_kick(&s, (1.0 - 2.0 * l2) * e);
            md_drift(&s, 0.5 * e);
        }
        md_kick(&s, l2 * e);
        break;
    case 4:   /* OMF_4_slow (:195-237) */
        for (int k = 0; k < n; ++k) { md_kick(&s, a4 * e); md_omf4_middle(&s, e, 0); md_kick(&s, a4 * e); }
        break;
    case 5:   /* OMF_4 (:241-294) */
        md_kick(&s, a4 * e);
        md_omf4_middle(&s, e, 0);
        for (int k = 0; k < n - 1; ++k) { md_kick(&s, 2.0 * a4 * e); md_omf4_middle(&s, e, 0); }
        md_kick(&s, a4 * e);
        break;
    case 6:   /* Leapfrog_friction_slow (:74-116) */
    case 7:   /* OMF_4_friction_slow (:298-376) */
    {
        double fric = 0.01;
        const int omf4 = integrator == 7, half = n / 2;
        for (int k = 0; k < half; ++k) md_friction_step(&s, omf4, e, &fric, 0);
        if (n % 2 != 0) md_friction_step(&s, omf4, e, &fric, 1);
        else fric = -fric;
        for (int k = 0; k < half; ++k) md_friction_step(&s, omf4, e, &fric, 0);
        break;
    }
    case 8:   /* Leapfrog_OMF_4 (hmc_metadynamics.hpp:28-83) */
        md_kick_metad(&s, 0.5 * e);
        for (int k = 0; k < n; ++k)
        {
            md_kick_gauge(&s, a4 * e); md_omf4_middle(&s, e, 1); md_kick_gauge(&s, a4 * e);
            md_kick_metad(&s, k < n - 1 ? e : 0.5 * e);
        }
        break;
    case 9:   /* OMF_2_OMF_4_slow (:85-143) */
        for (int k = 0; k < n; ++k)
        {
            md_kick_metad(&s, l2 * e);
            md_kick_gauge(&s, a4 * e); md_omf4_middle(&s, e, 1); md_kick_gauge(&s, a4 * e);
            md_kick_metad(&s, (1.0 - 2.0 * l2) * e);
            md_kick_gauge(&s, a4 * e); md_omf4_middle(&s, e, 1); md_kick_gauge(&s, a4 * e);
            md_kick_metad(&s, l2 * e);
        }
        break;
    case 10:  /* OMF_2_OMF_4 (:145-237): the inner OMF4 at half steps */
        md_kick_metad(&s, l2 * e);
        for (int k = 0; k < n; ++k)
        {
            md_kick_gauge(&s, 0.5 * a4 * e); md_omf4_middle(&s, 0.5 * e, 1); md_kick_gauge(&s, 0.5 * a4 * e);
            md_kick_metad(&s, (1.0 - 2.0 * l2) * e);
            md_kick_gauge(&s, 0.5 * a4 * e); md_omf4_middle(&s, 0.5 * e, 1); md_kick_gauge(&s, 0.5 * a4 * e);
            md_kick_metad(&s, k < n - 1 ? 2.0 * l2 * e : l2 * e);
        }
        break;
    default:
        break;
    }
    *h_new = md_energy(&s);
    free(s.F);
}

/* ParityUpdate (updates/parity_update.hpp:22-47) */
void or_parity_update(const int ext[4], double* U)
{
    Geo g = geo(ext);
    size_t n = (size_t)g.V * 72;
    double* c = (double*)malloc(n * sizeof(double));
    memcpy(c, U, n * sizeof(double));
    const int Nx = ext[1], Ny = ext[2], Nz = ext[3];
    for (int t = 0; t < ext[0]; ++t)
        for (int x = 0; x < Nx; ++x)
            for (int y = 0; y < Ny; ++y)
                for (int z = 0; z < Nz; ++z)
                {
                    const long site = (((long)t * Nx + x) * Ny + y) * Nz + z;
                    const int rx = Nx - x - 1, ry = Ny - y - 1, rz = Nz - z - 1;
                    const int rxm = (rx - 1 + Nx) % Nx, rym = (ry - 1 + Ny) % Ny, rzm = (rz - 1 + Nz) % Nz;
#define SITE(tt, xx, yy, zz) ((((long)(tt) * Nx + (xx)) * Ny + (yy)) * Nz + (zz))
                    M3 m0 = ld(c, SITE(t, rx, ry, rz), 0);
                    M3 m1 = dag(ld(c, SITE(t, rxm, ry, rz), 1));
                    M3 m2 = dag(ld(c, SITE(t, rx, rym, rz), 2));
                    M3 m3 = dag(ld(c, SITE(t, rx, ry, rzm), 3));
#undef SITE
                    st(U, site, 0, &m0);
                    st(U, site, 1, &m1);
                    st(U, site, 2, &m2);
                    st(U, site, 3, &m3);
                }
    free(c);
}

/* ---------------------------------------------------------------- bias potential */
/* MetaBiasPotential (metadynamics.hpp:60-187), well-tempered deposits */
or_bias* or_bias_create(double cv_min, double cv_max, int bins, double weight, double width, double wt, double thr)
{
    if (!(cv_min < cv_max) || bins <= 0) return NULL;
    or_bias* b = (or_bias*)calloc(1, sizeof(or_bias) + sizeof(double) * (size_t)bins);
    b->cv_min = cv_min; b->cv_max = cv_max; b->bins = bins;
    b->bin_width = (cv_max - cv_min) / bins; b->bin_width_inv = 1.0 / b->bin_width;
    b->weight = weight; b->width = width; b->wt = wt; b->thr = thr;
    return b;
}

void or_bias_destroy(or_bias* b) { free(b); }

void or_bias_update(or_bias* b, double cv)
{
    double wis = 1.0 / (b->width * b->width);
    for (int i = 0; i <= b->bins; ++i)
    {
        double d = cv - (b->cv_min + i * b->bin_width);
        b->grid[i] += b->weight * exp(-0.5 * wis * d * d - b->grid[i] / b->wt);
    }
}

/* The Gaussian-free binned deposit (semantics not in the reference, which deposits Gaussians;
 * parity unpinned): with x = (cv - cv_min) / bin_width the grid points floor(x) and
 * floor(x) + 1 receive weight (1 - frac(x)) and weight frac(x), each times
 * exp(-V_point / wt) (the reference's per-point well-tempering, metadynamics.hpp:116-118).
 * Out-of-range CVs deposit nothing. */
void or_bias_update_binned(or_bias* b, double cv)
{
    double x, a, v0, v1;
    int i;
    if (!(cv >= b->cv_min && cv < b->cv_max)) return;
    x = (cv - b->cv_min) / b->bin_width;
    i = (int)floor(x);
    if (i < 0) i = 0;
    if (i > b->bins - 1) i = b->bins - 1;
    a = x - (double)i;
    if (a < 0.0) a = 0.0;
    if (a > 1.0) a = 1.0;
    v0 = b->grid[i];
    v1 = b->grid[i + 1];
    b->grid[i] = v0 + b->weight * (1.0 - a) * exp(-v0 / b->wt);
    b->grid[i + 1] = v1 + b->weight * a * exp(-v1 / b->wt);
}

void or_bias_update_symmetric(or_bias* b, double cv)
{
    or_bias_update(b, cv);
    or_bias_update(b, -cv);
}

double or_bias_potential(const or_bias* b, double cv)
{
    int i = (int)floor((cv - b->cv_min) * b->bin_width_inv);
    if ((unsigned)i < (unsigned)b->bins)
    {
        double a = (cv - (b->cv_min + i * b->bin_width)) * b->bin_width_inv;
        return b->grid[i] * (1.0 - a) + a * b->grid[i + 1];
    }
    if (i < 0)
    {
        double d = cv - b->cv_min;
        return b->grid[0] + b->thr * d * d;
    }
    double d = cv - b->cv_max;
    return b->grid[b->bins] + b->thr * d * d;
}

double or_bias_derivative(const or_bias* b, double cv)
{
    double h = 0.5 * b->bin_width;
    return b->bin_width_inv * (or_bias_potential(b, cv + h) - or_bias_potential(b, cv - h));
}

/* ---------------------------------------------------------------- BMW configuration files */
/* Payload of the BMW format (IO/config_io/bmw_format.hpp:27-47, :294-394, :564-645): sites in
 * t, z, y, x order (x fastest), per site the directions x, y, z, t (reference mu = 1, 2, 3, 0),
 * per link the first two rows (full: all three), row-major, re then im, as big-endian doubles.
 * Checksum_Adler64 (bmw_format.hpp:63-97) runs over the native 64-bit words of every site block
 * of 4 * nw words: d0, d1 = high and low halves; A += d0 + d1; B += (2 + revi d0 + (revi - 1) d1)
 * mod p with revi = (V - block) * 2 * (4 nw) - 2 * word, all in wrapping 64-bit arithmetic;
 * final = ((B mod p) << 32) + (A + 1) mod p, p = 4294967291. */
static const uint64_t ADLER64_PRIME = 4294967291ULL;

static uint64_t bswap64(uint64_t v)
{
    uint64_t r = 0;
    for (int k = 0; k < 8; ++k) r |= ((v >> (8 * k)) & 0xFFULL) << (8 * (7 - k));
    return r;
}

static void adler64_block(const uint64_t* w, uint64_t block, uint64_t nblocks, int bs, uint64_t* A, uint64_t* B)
{
    uint64_t sa = 0, sb = 0;
    uint64_t revi = (nblocks - block) * (uint64_t)(2 * bs);
    for (int i = 0; i < bs; ++i)
    {
        uint64_t d0 = w[i] >> 32, d1 = w[i] & 0xFFFFFFFFULL;
        sa += d0 + d1;
        sb += (2 + revi * d0 + (revi - 1) * d1) % ADLER64_PRIME;
        revi -= 2;
    }
    *A = (*A + sa) % ADLER64_PRIME;
    *B = (*B + sb) % ADLER64_PRIME;
}

static uint64_t adler64_final(uint64_t A, uint64_t B)
{
    return ((B % ADLER64_PRIME) << 32) + (A + 1) % ADLER64_PRIME;
}

uint64_t or_bmw_encode(const int ext[4], const double* U, int full, unsigned char* payload)
{
    const int nw = full ? 18 : 12;
    Geo g = geo(ext);
    uint64_t A = 0, B = 0;
    uint64_t buf[4 * 18];
    const int Nt = ext[0], Nx = ext[1], Ny = ext[2], Nz = ext[3];
    for (int t = 0; t < Nt; ++t)
        for (int z = 0; z < Nz; ++z)
            for (int y = 0; y < Ny; ++y)
                for (int x = 0; x < Nx; ++x)
                {
                    const int c[4] = { t, x, y, z };
                    const long s = site_of(&g, c);
                    for (int dp = 0; dp < 4; ++dp)
                    {
                        const int mu = (dp + 1) % 4;
                        memcpy(buf + dp * nw, U + 18 * (4 * s + mu), sizeof(double) * (size_t)nw);
                    }
                    const uint64_t block = (((uint64_t)t * Nz + z) * Ny + y) * Nx + x;
                    adler64_block(buf, block, (uint64_t)g.V, 4 * nw, &A, &B);
                    if (payload)
                        for (int k = 0; k < 4 * nw; ++k)
                        {
                            uint64_t be = bswap64(buf[k]);
                            memcpy(payload + (block * 4 * nw + (uint64_t)k) * 8, &be, 8);
                        }
                }
    return adler64_final(A, B);
}

uint64_t or_bmw_decode(const int ext[4], const unsigned char* payload, int full, double* U)
{
    const int nw = full ? 18 : 12;
    Geo g = geo(ext);
    uint64_t A = 0, B = 0;
    uint64_t buf[4 * 18];
    const int Nt = ext[0], Nx = ext[1], Ny = ext[2], Nz = ext[3];
    for (int t = 0; t < Nt; ++t)
        for (int z = 0; z < Nz; ++z)
            for (int y = 0; y < Ny; ++y)
                for (int x = 0; x < Nx; ++x)
                {
                    const uint64_t block = (((uint64_t)t * Nz + z) * Ny + y) * Nx + x;
                    for (int k = 0; k < 4 * nw; ++k)
                    {
                        uint64_t be;
                        memcpy(&be, payload + (block * 4 * nw + (uint64_t)k) * 8, 8);
                        buf[k] = bswap64(be);
                    }
                    adler64_block(buf, block, (uint64_t)g.V, 4 * nw, &A, &B);
                    const int c[4] = { t, x, y, z };
                    const long s = site_of(&g, c);
                    for (int dp = 0; dp < 4; ++dp)
                    {
                        const int mu = (dp + 1) % 4;
                        double* p = U + 18 * (4 * s + mu);
                        memset(p, 0, sizeof(double) * 18);
                        memcpy(p, buf + dp * nw, sizeof(double) * (size_t)nw);
                        if (!full)
                        {
                            /* ReconstructMatBMW + SU3::Projection::RestoreLastRow (bmw_format.hpp:131-143, :247-250) */
                            M3 m = ld(U, s, mu);
                            m.m[2][0] = conj(m.m[0][1] * m.m[1][2] - m.m[0][2] * m.m[1][1]);
                            m.m[2][1] = conj(m.m[0][2] * m.m[1][0] - m.m[0][0] * m.m[1][2]);
                            m.m[2][2] = conj(m.m[0][0] * m.m[1][1] - m.m[0][1] * m.m[1][0]);
                            st(U, s, mu, &m);
                        }
                    }
                }
    return adler64_final(A, B);
}

/* ---------------------------------------------------------------- measurement bundle */
/* The observables SU3_main.cpp:89-235 measures on every smearing level. */

/* TopChargeCloverTimeslice and EnergyDensity::CloverTimeslice (topological_charge.hpp:338-364,
 * field_strength_tensor.hpp:178-195) for every t: the densities of or_topcharge_clover and
 * or_energy_clover summed over one timeslice, with their normalisations (sum over t = total). */
void or_clover_timeslices(const int ext[4], const double* U, double* q_t, double* e_t)
{
    Geo g = geo(ext);
    for (int t = 0; t < ext[0]; ++t) q_t[t] = e_t[t] = 0.0;
    for (long s = 0; s < g.V; ++s)
    {
        int c[4];
        coords(&g, s, c);
        M3 F[4][4];
        double e = 0.0;
        for (int mu = 0; mu < 4; ++mu)
            for (int nu = mu + 1; nu < 4; ++nu)
            {
                M3 cl = clover(&g, U, s, mu, nu);
                F[mu][nu] = sub(cl, dag(cl));
                M3 f = scl(-I / 4.0, scl(0.5, F[mu][nu]));
                cd tt = tr(f) / 3.0;
                for (int i = 0; i < 3; ++i) f.m[i][i] -= tt;
                e += creal(tr(mul(f, f)));
            }
        double q = creal(tr(sub(add(mul(F[0][1], F[2][3]), mul(F[0][3], F[1][2])), mul(F[0][2], F[1][3]))));
        q_t[c[0]] += -1.0 / (64.0 * 4.0 * PI * PI) * q;
        e_t[c[0]] += e / (double)g.V;
    }
}

/* TopChargePlaquette (topological_charge.hpp:366-416): F = -i (P - P^dag) from the forward
 * plaquettes, Q = 1/(16 pi^2) sum Re tr(F01 F23 + F02 F31 + F03 F12) */
double or_topcharge_plaquette(const int ext[4], const double* U)
{
    Geo g = geo(ext);
    double q = 0.0;
    for (long s = 0; s < g.V; ++s)
    {
        M3 F[4][4];
        for (int mu = 0; mu < 4; ++mu)
            for (int nu = mu + 1; nu < 4; ++nu)
            {
                M3 p = plaquette(&g, U, s, mu, nu);
                F[mu][nu] = scl(-I, sub(p, dag(p)));
                F[nu][mu] = scl(-1.0, F[mu][nu]);
            }
        q += creal(tr(add(add(mul(F[0][1], F[2][3]), mul(F[0][2], F[3][1])), mul(F[0][3], F[1][2]))));
    }
    return 1.0 / (16.0 * PI * PI) * q;
}

/* Rectangular<2>::Action (actions/gauge/rectangular_action.hpp:61-94) with the 1x2 and 2x1
 * loops of wilson_loop.hpp:155-175 */
double or_rect_action(const int ext[4], const double* U, double beta, double c_plaq, double c_rect)
{
    Geo g = geo(ext);
    double sp = 0.0, sr = 0.0;
    for (long s = 0; s < g.V; ++s)
        for (int nu = 1; nu < 4; ++nu)
            for (int mu = 0; mu < nu; ++mu)
            {
                sp += creal(tr(plaquette(&g, U, s, mu, nu)));
                long smu = move(&g, s, mu, 1), snu = move(&g, s, nu, 1);
                long smu_nu = move(&g, smu, nu, 1), snu2 = move(&g, snu, nu, 1), smu2 = move(&g, smu, mu, 1);
                /* <1,2>: U_mu(x) U_nu(x+mu) U_nu(x+mu+nu) U_mu(x+2nu)^dag U_nu(x+nu)^dag U_nu(x)^dag */
                M3 r12 = mul(mul(mul(mul(mul(ld(U, s, mu), ld(U, smu, nu)), ld(U, smu_nu, nu)), dag(ld(U, snu2, mu))),
                                 dag(ld(U, snu, nu))), dag(ld(U, s, nu)));
                /* <2,1>: U_mu(x) U_mu(x+mu) U_nu(x+2mu) U_mu(x+mu+nu)^dag U_mu(x+nu)^dag U_nu(x)^dag */
                M3 r21 = mul(mul(mul(mul(mul(ld(U, s, mu), ld(U, smu, mu)), ld(U, smu2, nu)), dag(ld(U, smu_nu, mu))),
                                 dag(ld(U, snu, mu))), dag(ld(U, s, nu)));
                sr += creal(tr(r12)) + creal(tr(r21));
            }
    return beta * (c_plaq * (6.0 * g.V - sp / 3.0) + c_rect * (12.0 * g.V - sr / 3.0));
}

/* Line product C_mu(x) = U_mu(x) U_mu(x+mu) ... U_mu(x+(L-1)mu) */
static M3 line(const Geo* g, const double* U, long s, int mu, int L)
{
    M3 r = ld(U, s, mu);
    long t = s;
    for (int k = 1; k < L; ++k)
    {
        t = move(g, t, mu, 1);
        r = mul(r, ld(U, t, mu));
    }
    return r;
}

/* WilsonLoop<0, L, true> (observables/wilson_loop.hpp:63-124): square L x L loops in all six
 * planes, 1 - sum Re tr(C_mu(x) C_nu(x+L mu) C_mu(x+L nu)^dag C_nu(x)^dag) / (6 * 3 * V) */
double or_wilson_loop(const int ext[4], const double* U, int L)
{
    Geo g = geo(ext);
    double w = 0.0;
    for (long s = 0; s < g.V; ++s)
        for (int mu = 0; mu < 4; ++mu)
            for (int nu = mu + 1; nu < 4; ++nu)
            {
                long smu = s, snu = s;
                for (int k = 0; k < L; ++k)
                {
                    smu = move(&g, smu, mu, 1);
                    snu = move(&g, snu, nu, 1);
                }
                M3 m = mul(mul(mul(line(&g, U, s, mu, L), line(&g, U, smu, nu, L)), dag(line(&g, U, snu, mu, L))),
                           dag(line(&g, U, s, nu, L)));
                w += creal(tr(m));
            }
    return 1.0 - w / (18.0 * (double)g.V);
}

/* PolyakovLoop (observables/polyakov_loop.hpp:32-49): the trace of the product of the t links
 * over every spatial site, averaged over the spatial volume */
void or_polyakov_loop(const int ext[4], const double* U, double* re, double* im)
{
    cd p = 0.0;
    long vs = (long)ext[1] * ext[2] * ext[3];
    for (long k = 0; k < vs; ++k)
    {
        M3 m = id3();
        for (int t = 0; t < ext[0]; ++t) m = mul(m, ld(U, (long)t * vs + k, 0));
        p += tr(m);
    }
    *re = creal(p) / (double)vs;
    *im = cimag(p) / (double)vs;
}
