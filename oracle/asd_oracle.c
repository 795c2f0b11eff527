/* FP64 CPU oracle for the reference sLLG step.  TEST INFRASTRUCTURE ONLY:
 * loaded by tests/, __graft_entry__.smoke() and bench.py's CPU legs, never
 * by the product.  See asd_oracle.h for the semantics and the quirk flags.
 *
 * Arithmetic is scalar IEEE-754 double with no FMA contraction
 * (-ffp-contract=off); the operation order of every expression follows the
 * cited reference line so that, given the same inputs, results are
 * reproducible to the last bit by code written the same way.
 */
#include "asd_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

struct orc_ctx {
    uint32_t n;
    double *s, *es, *fn, *h, *hdemag, *det, *noise, *k[6], *hstag;
    double* h4s;                         /* llgCPU's separate four-spin field (CPU_SUM_ORDER only) */
    double *llgpf, *lambda, *sigma, *k1u, *k1udir;
    double k2perp, k2perpdir[3], k2par, k2pardir[3], k4perp, k4perpdirs[9], k4par, k4pardirs[9], basemm;
    int integrator;
    double rdt, applied[3], stag_scale;
    double pulse_amp, pulse_t0, pulse_sigma, dt, cur_scale;
    uint32_t nrep, *rep_off, *rep_stream;
    double* rep_T;
    int exch, full;
    uint32_t nnz, *xadj, *adjncy;
    double* csr;        /* nnz x 9 */
    uint32_t ndiag;
    int32_t* doff;
    double* dia;        /* 9 x ndiag x n */
    int lr;
    uint32_t mesh[3], nspec, update;
    uint32_t *mesh_xyz, *spec;
    double *nr, *w;
    uint32_t flags;
    int noise_mode;
    uint64_t seed;
    double* nbuf;
    size_t nbuf_len, nbuf_pos;
    uint32_t *q4ptr, *q4j, *q4k, *q4l;   /* four-spin quartets (CSR over spins), or NULL */
    double q4jq;
    int q4div3;
};

/* ------------------------------------------------------------------ */
/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
 * easy as 1, 2, 3", SC'11): 10 rounds of two 32x32->64 multiplies with the
 * published multipliers and Weyl key increments.                        */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; r++) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* Natural log from its atanh series, ln m = 2 sum f^(2k+1)/(2k+1) with
 * f=(m-1)/(m+1), after reducing x = m 2^e, m in [sqrt(1/2), sqrt(2)).
 * Only correctly rounded operations are used, so the value is identical on
 * any IEEE-754 machine that evaluates it in this order. */
double orc_log(double x) {
    int e;
    double m = frexp(x, &e);
    if (m < 0x1.6a09e667f3bcdp-1) { m = m * 2.0; e = e - 1; }
    double f = (m - 1.0) / (m + 1.0);
    double f2 = f * f;
    double p = 0x1.642c8590b2164p-5;            /* 1/23 */
    p = fma(p, f2, 0x1.8618618618618p-5);       /* 1/21 */
    p = fma(p, f2, 0x1.af286bca1af28p-5);       /* 1/19 */
    p = fma(p, f2, 0x1.e1e1e1e1e1e1ep-5);       /* 1/17 */
    p = fma(p, f2, 0x1.1111111111111p-4);       /* 1/15 */
    p = fma(p, f2, 0x1.3b13b13b13b14p-4);       /* 1/13 */
    p = fma(p, f2, 0x1.745d1745d1746p-4);       /* 1/11 */
    p = fma(p, f2, 0x1.c71c71c71c71cp-4);       /* 1/9 */
    p = fma(p, f2, 0x1.2492492492492p-3);       /* 1/7 */
    p = fma(p, f2, 0x1.999999999999ap-3);       /* 1/5 */
    p = fma(p, f2, 0x1.5555555555555p-2);       /* 1/3 */
    p = fma(p, f2, 1.0);
    double lnm = 2.0 * (f * p);
    return fma((double)e, 0x1.62e42fefa39efp-1, lnm);
}

/* sin and cos of 2*pi*u for u=(x+0.5)/2^32: octant reduction is exact
 * because 8u has at most 33 significant bits; Taylor series on [0, pi/4]. */
void orc_sincos_2pi(uint32_t x, double* sn, double* cs) {
    double v = ((double)x + 0.5) * 0x1p-29;     /* 8u, exact */
    double qd = floor(v);
    int q = (int)qd;
    double r = v - qd;                          /* exact */
    double psi = ((q & 1) ? (1.0 - r) : r) * 0x1.921fb54442d18p-1;
    double p2 = psi * psi;
    double sp = 0x1.2f49b46814157p-57;          /* 1/19! */
    sp = fma(sp, -p2, 0x1.952c77030ad4ap-49);   /* 1/17! */
    sp = fma(sp, -p2, 0x1.ae7f3e733b81fp-41);   /* 1/15! */
    sp = fma(sp, -p2, 0x1.6124613a86d09p-33);   /* 1/13! */
    sp = fma(sp, -p2, 0x1.ae64567f544e4p-26);   /* 1/11! */
    sp = fma(sp, -p2, 0x1.71de3a556c734p-19);   /* 1/9! */
    sp = fma(sp, -p2, 0x1.a01a01a01a01ap-13);   /* 1/7! */
    sp = fma(sp, -p2, 0x1.1111111111111p-7);    /* 1/5! */
    sp = fma(sp, -p2, 0x1.5555555555555p-3);    /* 1/3! */
    sp = fma(sp, -p2, 1.0);
    double s = psi * sp;
    double cp = 0x1.6827863b97d97p-53;          /* 1/18! */
    cp = fma(cp, -p2, 0x1.ae7f3e733b81fp-45);   /* 1/16! */
    cp = fma(cp, -p2, 0x1.93974a8c07c9dp-37);   /* 1/14! */
    cp = fma(cp, -p2, 0x1.1eed8eff8d898p-29);   /* 1/12! */
    cp = fma(cp, -p2, 0x1.27e4fb7789f5cp-22);   /* 1/10! */
    cp = fma(cp, -p2, 0x1.a01a01a01a01ap-16);   /* 1/8! */
    cp = fma(cp, -p2, 0x1.6c16c16c16c17p-10);   /* 1/6! */
    cp = fma(cp, -p2, 0x1.5555555555555p-5);    /* 1/4! */
    cp = fma(cp, -p2, 0x1.0000000000000p-1);    /* 1/2! */
    double c = fma(cp, -p2, 1.0);
    switch (q) {
    case 0: *sn = s;  *cs = c;  break;
    case 1: *sn = c;  *cs = s;  break;
    case 2: *sn = c;  *cs = -s; break;
    case 3: *sn = s;  *cs = -c; break;
    case 4: *sn = -s; *cs = -c; break;
    case 5: *sn = -c; *cs = -s; break;
    case 6: *sn = -c; *cs = s;  break;
    default: *sn = -s; *cs = c; break;
    }
}

/* Three N(0,1) deviates for (stream, spin, step): one Philox call with
 * counter (spin, step_lo, step_hi, stream) and key (seed_lo, seed_hi), then
 * Box-Muller on the pairs (u0,u1) -> x,y and (u2,u3) -> z. */
void orc_thermal_normals(uint64_t seed, uint32_t stream, uint32_t spin, uint64_t step, double out[3]) {
    uint32_t ctr[4] = {spin, (uint32_t)step, (uint32_t)(step >> 32), stream};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t x[4];
    orc_philox4x32_10(ctr, key, x);
    double u0 = ((double)x[0] + 0.5) * 0x1p-32;
    double u2 = ((double)x[2] + 0.5) * 0x1p-32;
    double r0 = sqrt(-2.0 * orc_log(u0));
    double r2 = sqrt(-2.0 * orc_log(u2));
    double s1, c1, s3, c3;
    orc_sincos_2pi(x[1], &s1, &c1);
    orc_sincos_2pi(x[3], &s3, &c3);
    out[0] = r0 * c1;
    out[1] = r0 * s1;
    out[2] = r2 * c3;
}

/* Single-precision variant (the FP32 form's generator): uniforms (float(x)+0.5)/2^32,
 * octant from the top 3 bits, ln to f^11, sin to psi^11, cos to psi^12, float fma. */
static float logf_series(float x) {
    int e;
    float m = frexpf(x, &e);
    if (m < 0x1.6a09e6p-1f) { m = m * 2.0f; e = e - 1; }
    const float f = (m - 1.0f) / (m + 1.0f);
    const float f2 = f * f;
    float p = 0x1.745d18p-4f;
    p = fmaf(p, f2, 0x1.c71c72p-4f);
    p = fmaf(p, f2, 0x1.24924ap-3f);
    p = fmaf(p, f2, 0x1.99999ap-3f);
    p = fmaf(p, f2, 0x1.555556p-2f);
    p = fmaf(p, f2, 1.0f);
    const float lnm = 2.0f * (f * p);
    return fmaf((float)e, 0x1.62e430p-1f, lnm);
}

static void sincosf_series(uint32_t x, float* sn, float* cs) {
    const int q = (int)(x >> 29);
    const float r = ((float)(x & 0x1FFFFFFFu) + 0.5f) * 0x1p-29f;
    const float psi = ((q & 1) ? (1.0f - r) : r) * 0x1.921fb6p-1f;
    const float mp2 = -(psi * psi);
    float sp = 0x1.ae6456p-26f;
    sp = fmaf(sp, mp2, 0x1.71de3ap-19f);
    sp = fmaf(sp, mp2, 0x1.a01a02p-13f);
    sp = fmaf(sp, mp2, 0x1.111112p-7f);
    sp = fmaf(sp, mp2, 0x1.555556p-3f);
    sp = fmaf(sp, mp2, 1.0f);
    const float s = psi * sp;
    float cp = 0x1.1eed8ep-29f;
    cp = fmaf(cp, mp2, 0x1.27e4fcp-22f);
    cp = fmaf(cp, mp2, 0x1.a01a02p-16f);
    cp = fmaf(cp, mp2, 0x1.6c16c2p-10f);
    cp = fmaf(cp, mp2, 0x1.555556p-5f);
    cp = fmaf(cp, mp2, 0x1.000000p-1f);
    const float c = fmaf(cp, mp2, 1.0f);
    switch (q) {
    case 0: *sn = s;  *cs = c;  break;
    case 1: *sn = c;  *cs = s;  break;
    case 2: *sn = c;  *cs = -s; break;
    case 3: *sn = s;  *cs = -c; break;
    case 4: *sn = -s; *cs = -c; break;
    case 5: *sn = -c; *cs = -s; break;
    case 6: *sn = -c; *cs = s;  break;
    default: *sn = -s; *cs = c; break;
    }
}

void orc_thermal_normals_f(uint64_t seed, uint32_t stream, uint32_t spin, uint64_t step, float out[3]) {
    uint32_t ctr[4] = {spin, (uint32_t)step, (uint32_t)(step >> 32), stream};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t x[4];
    orc_philox4x32_10(ctr, key, x);
    const float u0 = ((float)x[0] + 0.5f) * 0x1p-32f;
    const float u2 = ((float)x[2] + 0.5f) * 0x1p-32f;
    const float r0 = sqrtf(-2.0f * logf_series(u0));
    const float r2 = sqrtf(-2.0f * logf_series(u2));
    float s1, c1, s3, c3;
    sincosf_series(x[1], &s1, &c1);
    sincosf_series(x[3], &s3, &c3);
    out[0] = r0 * c1;
    out[1] = r0 * s1;
    out[2] = r2 * c3;
}

/* MWC1616 and Marsaglia's polar method, restating src/random.cpp:17-64. */
static uint32_t mwc_x = 1, mwc_y = 1;
static int mwc_sw = 0;
static double mwc_n2 = 0.0;
void orc_mwc_seed(uint32_t a, uint32_t b) { mwc_x = a; mwc_y = b; mwc_sw = 0; }
static uint32_t mwc_next(void) {
    mwc_x = 18000u * (mwc_x & 0xFFFFu) + (mwc_x >> 16);
    mwc_y = 30903u * (mwc_y & 0xFFFFu) + (mwc_y >> 16);
    return (mwc_x << 16) + (mwc_y & 0xFFFFu);
}
double orc_mwc_rand(void) { return mwc_next() * (1.0 / 4294967295.0); }
double orc_mwc_normal(void) {
    if (!mwc_sw) {
        double w, x1, x2;
        for (;;) {
            const double u = 1.0 - mwc_next() * (1.0 / 4294967295.0);
            const double v = 1.0 - mwc_next() * (1.0 / 4294967295.0);
            x1 = 2.0 * u - 1.0;
            x2 = 2.0 * v - 1.0;
            w = x1 * x1 + x2 * x2;
            if (w < 1.0) break;
        }
        w = sqrt((-2.0 * log(w)) / w);
        mwc_n2 = w * x2;
        mwc_sw = 1;
        return w * x1;
    }
    mwc_sw = 0;
    return mwc_n2;
}

/* ------------------------------------------------------------------ */
static double* dalloc(size_t n) { return (double*)calloc(n ? n : 1, sizeof(double)); }

orc_ctx* orc_create(uint32_t n) {
    orc_ctx* c = (orc_ctx*)calloc(1, sizeof(orc_ctx));
    c->n = n;
    c->s = dalloc(3 * (size_t)n); c->es = dalloc(3 * (size_t)n); c->fn = dalloc(3 * (size_t)n);
    c->h = dalloc(3 * (size_t)n); c->hdemag = dalloc(3 * (size_t)n); c->det = dalloc(3 * (size_t)n);
    c->h4s = dalloc(3 * (size_t)n);
    c->noise = dalloc(3 * (size_t)n); c->hstag = dalloc(3 * (size_t)n);
    for (int k = 0; k < 6; k++) c->k[k] = dalloc(3 * (size_t)n);
    c->llgpf = dalloc(n); c->lambda = dalloc(n); c->sigma = dalloc(n); c->k1u = dalloc(n);
    c->k1udir = dalloc(3 * (size_t)n);
    c->nrep = 1;
    c->rep_off = (uint32_t*)calloc(2, sizeof(uint32_t)); c->rep_off[1] = n;
    c->rep_stream = (uint32_t*)calloc(1, sizeof(uint32_t));
    c->rep_T = dalloc(1);
    c->stag_scale = 1.0;
    c->basemm = 1.0;
    c->update = 1;
    return c;
}

static void freep(void* p) { if (p) free(p); }
void orc_destroy(orc_ctx* c) {
    if (!c) return;
    freep(c->s); freep(c->es); freep(c->fn); freep(c->h); freep(c->hdemag); freep(c->det); freep(c->h4s);
    freep(c->noise); freep(c->hstag);
    for (int k = 0; k < 6; k++) freep(c->k[k]);
    freep(c->llgpf); freep(c->lambda); freep(c->sigma); freep(c->k1u); freep(c->k1udir);
    freep(c->rep_off); freep(c->rep_stream); freep(c->rep_T);
    freep(c->xadj); freep(c->adjncy); freep(c->csr); freep(c->doff); freep(c->dia);
    freep(c->mesh_xyz); freep(c->spec); freep(c->nr); freep(c->w); freep(c->nbuf);
    freep(c->q4ptr); freep(c->q4j); freep(c->q4k); freep(c->q4l);
    free(c);
}

int orc_set_material(orc_ctx* c, const double* llgpf, const double* lambda, const double* sigma,
                     const double* k1u, const double* k1udir) {
    uint32_t n = c->n;
    memcpy(c->llgpf, llgpf, n * sizeof(double));
    memcpy(c->lambda, lambda, n * sizeof(double));
    memcpy(c->sigma, sigma, n * sizeof(double));
    if (k1u) memcpy(c->k1u, k1u, n * sizeof(double));
    if (k1udir) memcpy(c->k1udir, k1udir, 3 * (size_t)n * sizeof(double));
    return 0;
}

int orc_set_global_anis(orc_ctx* c, double k2perp, const double* k2perpdir, double k2par, const double* k2pardir,
                        double k4perp, const double* k4perpdirs, double k4par, const double* k4pardirs, double basemm) {
    c->k2perp = k2perp; c->k2par = k2par; c->k4perp = k4perp; c->k4par = k4par; c->basemm = basemm;
    for (int a = 0; a < 3; a++) {
        c->k2perpdir[a] = k2perpdir ? k2perpdir[a] : 0.0;
        c->k2pardir[a] = k2pardir ? k2pardir[a] : 0.0;
    }
    for (int a = 0; a < 9; a++) {
        c->k4perpdirs[a] = k4perpdirs ? k4perpdirs[a] : 0.0;
        c->k4pardirs[a] = k4pardirs ? k4pardirs[a] : 0.0;
    }
    return 0;
}

int orc_set_dynamics(orc_ctx* c, int integrator, double rdt, const double* applied) {
    if (integrator < 0 || integrator > 2) return -1;
    c->integrator = integrator;
    c->rdt = rdt;
    for (int a = 0; a < 3; a++) c->applied[a] = applied ? applied[a] : 0.0;
    return 0;
}

int orc_set_replicas(orc_ctx* c, uint32_t nrep, const uint32_t* off, const double* T, const uint32_t* stream) {
    if (nrep == 0 || off[0] != 0 || off[nrep] != c->n) return -1;
    freep(c->rep_off); freep(c->rep_T); freep(c->rep_stream);
    c->nrep = nrep;
    c->rep_off = (uint32_t*)malloc((nrep + 1) * sizeof(uint32_t));
    c->rep_T = dalloc(nrep);
    c->rep_stream = (uint32_t*)malloc(nrep * sizeof(uint32_t));
    memcpy(c->rep_off, off, (nrep + 1) * sizeof(uint32_t));
    memcpy(c->rep_T, T, nrep * sizeof(double));
    for (uint32_t r = 0; r < nrep; r++) c->rep_stream[r] = stream ? stream[r] : r;
    return 0;
}

int orc_set_csr(orc_ctx* c, int full, uint32_t nnz, const uint32_t* xadj, const uint32_t* adjncy, const double* val9) {
    freep(c->xadj); freep(c->adjncy); freep(c->csr);
    c->exch = ORC_EXCH_CSR; c->full = full; c->nnz = nnz;
    c->xadj = (uint32_t*)malloc((c->n + 1) * sizeof(uint32_t));
    c->adjncy = (uint32_t*)malloc((nnz ? nnz : 1) * sizeof(uint32_t));
    c->csr = dalloc(9 * (size_t)nnz);
    memcpy(c->xadj, xadj, (c->n + 1) * sizeof(uint32_t));
    memcpy(c->adjncy, adjncy, nnz * sizeof(uint32_t));
    memcpy(c->csr, val9, 9 * (size_t)nnz * sizeof(double));
    return 0;
}

int orc_set_dia(orc_ctx* c, int full, uint32_t ndiag, const int32_t* offsets, const double* val9) {
    freep(c->doff); freep(c->dia);
    c->exch = ORC_EXCH_DIA; c->full = full; c->ndiag = ndiag;
    c->doff = (int32_t*)malloc((ndiag ? ndiag : 1) * sizeof(int32_t));
    c->dia = dalloc(9 * (size_t)ndiag * c->n);
    memcpy(c->doff, offsets, ndiag * sizeof(int32_t));
    memcpy(c->dia, val9, 9 * (size_t)ndiag * c->n * sizeof(double));
    return 0;
}

int orc_set_site_field(orc_ctx* c, const double* hstag, double scale) {
    if (hstag) memcpy(c->hstag, hstag, 3 * (size_t)c->n * sizeof(double));
    else memset(c->hstag, 0, 3 * (size_t)c->n * sizeof(double));
    c->stag_scale = scale;
    return 0;
}

int orc_set_longrange(orc_ctx* c, int mode, const uint32_t* mesh_dims, const uint32_t* mesh_xyz,
                      uint32_t nspec, const uint32_t* spec, const double* nr, const double* w, uint32_t update) {
    freep(c->mesh_xyz); freep(c->spec); freep(c->nr); freep(c->w);
    c->mesh_xyz = NULL; c->spec = NULL; c->nr = NULL; c->w = NULL;
    c->lr = mode;
    if (mode == ORC_LR_NONE) return 0;
    for (int a = 0; a < 3; a++) c->mesh[a] = mesh_dims[a];
    c->nspec = nspec ? nspec : 1;
    c->update = update ? update : 1;
    size_t p = (size_t)c->mesh[0] * c->mesh[1] * c->mesh[2];
    c->mesh_xyz = (uint32_t*)malloc(3 * (size_t)c->n * sizeof(uint32_t));
    memcpy(c->mesh_xyz, mesh_xyz, 3 * (size_t)c->n * sizeof(uint32_t));
    c->spec = (uint32_t*)calloc(c->n, sizeof(uint32_t));
    if (spec) memcpy(c->spec, spec, c->n * sizeof(uint32_t));
    size_t nn = (size_t)c->nspec * c->nspec * 9 * p;
    c->nr = dalloc(nn);
    memcpy(c->nr, nr, nn * sizeof(double));
    c->w = dalloc(c->n);
    for (uint32_t i = 0; i < c->n; i++) c->w[i] = w ? w[i] : 1.0;
    return 0;
}

int orc_set_flags(orc_ctx* c, uint32_t flags) { c->flags = flags; return 0; }

int orc_set_noise(orc_ctx* c, int mode, uint64_t seed, uint32_t mwc_a, uint32_t mwc_b,
                  const double* buf, size_t buf_len) {
    c->noise_mode = mode;
    c->seed = seed;
    if (mode == ORC_NOISE_MWC) orc_mwc_seed(mwc_a, mwc_b);
    freep(c->nbuf); c->nbuf = NULL; c->nbuf_len = 0; c->nbuf_pos = 0;
    if (mode == ORC_NOISE_BUFFER) {
        c->nbuf = dalloc(buf_len);
        memcpy(c->nbuf, buf, buf_len * sizeof(double));
        c->nbuf_len = buf_len;
    }
    return 0;
}

static void normalise(double v[3]);

/* Spins are normalised on entry, s/|s| with |s| = sqrt(x*x+y*y+z*z), as the
 * reference does for spins read from a file (src/spins.cpp:388-392). */
int orc_set_spins(orc_ctx* c, const double* s) {
    for (uint32_t i = 0; i < c->n; i++) {
        double v[3] = {s[3 * (size_t)i], s[3 * (size_t)i + 1], s[3 * (size_t)i + 2]};
        normalise(v);
        memcpy(c->s + 3 * (size_t)i, v, sizeof(v));
    }
    return 0;
}
int orc_get_spins(const orc_ctx* c, double* s) { memcpy(s, c->s, 3 * (size_t)c->n * sizeof(double)); return 0; }
int orc_get_det_field(const orc_ctx* c, double* h) { memcpy(h, c->det, 3 * (size_t)c->n * sizeof(double)); return 0; }

/* ------------------------------------------------------------------ */
/* Exchange sums.  GPU order: dot[co] += val*S one term at a time
 * (src/cufields.cu:192-199, 222-239, 109-125, 150-168); CPU order: the three
 * products of a row summed first (src/matrix_mul_cpu.cpp:59-61,104-106). */
static void exch_sum(const orc_ctx* c, const double* src, uint32_t i, double dot[3]) {
    const int cpu = (c->flags & ORC_CPU_SUM_ORDER) != 0;
    const int zz_from_yy = (c->flags & ORC_GPU_DZZ_FROM_DYY) != 0;
    dot[0] = dot[1] = dot[2] = 0.0;
    if (c->exch == ORC_EXCH_CSR) {
        for (uint32_t k = c->xadj[i]; k < c->xadj[i + 1]; k++) {
            const uint32_t j = c->adjncy[k];
            const double* v = c->csr + 9 * (size_t)k;
            const double* sj = src + 3 * (size_t)j;
            double vv[9];
            memcpy(vv, v, sizeof(vv));
            if (zz_from_yy) vv[8] = vv[4];
            if (!c->full) {
                dot[0] += vv[0] * sj[0];
                dot[1] += vv[4] * sj[1];
                dot[2] += vv[8] * sj[2];
            } else if (cpu) {
                dot[0] += (vv[0] * sj[0] + vv[1] * sj[1] + vv[2] * sj[2]);
                dot[1] += (vv[3] * sj[0] + vv[4] * sj[1] + vv[5] * sj[2]);
                dot[2] += (vv[6] * sj[0] + vv[7] * sj[1] + vv[8] * sj[2]);
            } else {
                for (int co = 0; co < 3; co++)
                    for (int ro = 0; ro < 3; ro++) dot[co] += vv[3 * co + ro] * sj[ro];
            }
        }
    } else if (c->exch == ORC_EXCH_DIA) {
        const size_t m = (size_t)c->ndiag * c->n;
        for (uint32_t d = 0; d < c->ndiag; d++) {
            const int64_t col = (int64_t)i + c->doff[d];
            const size_t a = (size_t)d * c->n + i;
            if (col < 0 || col >= (int64_t)c->n) continue;
            const double* sj = src + 3 * (size_t)col;
            double vv[9];
            for (int q = 0; q < 9; q++) vv[q] = c->dia[(size_t)q * m + a];
            if (zz_from_yy) vv[8] = vv[4];
            if (!c->full) {
                dot[0] += vv[0] * sj[0];
                dot[1] += vv[4] * sj[1];
                dot[2] += vv[8] * sj[2];
            } else if (cpu) {
                dot[0] += (vv[0] * sj[0] + vv[1] * sj[1] + vv[2] * sj[2]);
                dot[1] += (vv[3] * sj[0] + vv[4] * sj[1] + vv[5] * sj[2]);
                dot[2] += (vv[6] * sj[0] + vv[7] * sj[1] + vv[8] * sj[2]);
            } else {
                for (int co = 0; co < 3; co++)
                    for (int ro = 0; ro < 3; ro++) dot[co] += vv[3 * co + ro] * sj[ro];
            }
        }
    }
}

/* Long-range field by direct summation over the periodic padded mesh: the
 * cyclic convolution that IFFT(N_k FFT(w S))/P evaluates
 * (src/cufields.cu:248-430, src/cuda.cu:47-60,65-76). */
static void longrange_field(const orc_ctx* c, const double* src, double* out) {
    const uint32_t n0 = c->mesh[0], n1 = c->mesh[1], n2 = c->mesh[2];
    const size_t p = (size_t)n0 * n1 * n2;
    const uint32_t ns = c->nspec;
    for (uint32_t i = 0; i < c->n; i++) {
        const uint32_t* xi = c->mesh_xyz + 3 * (size_t)i;
        const uint32_t si = c->spec[i];
        double acc[3] = {0.0, 0.0, 0.0};
        for (uint32_t j = 0; j < c->n; j++) {
            const uint32_t* xj = c->mesh_xyz + 3 * (size_t)j;
            const uint32_t sj = c->spec[j];
            const uint32_t dx = (xi[0] + n0 - xj[0]) % n0;
            const uint32_t dy = (xi[1] + n1 - xj[1]) % n1;
            const uint32_t dz = (xi[2] + n2 - xj[2]) % n2;
            const size_t cell = ((size_t)dx * n1 + dy) * n2 + dz;
            const double wj = c->w[j];
            const double m[3] = {src[3 * (size_t)j] * wj, src[3 * (size_t)j + 1] * wj, src[3 * (size_t)j + 2] * wj};
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++)
                    acc[a] += c->nr[((((size_t)si * ns + sj) * 3 + a) * 3 + b) * p + cell] * m[b];
        }
        out[3 * (size_t)i] = acc[0];
        out[3 * (size_t)i + 1] = acc[1];
        out[3 * (size_t)i + 2] = acc[2];
    }
}

/* CH += four-spin field, accumulated from zero per spin in quartet order:
 * cufields::CSpMV_CSR_FourSpin (src/cufields.cu:59-90), launched after the SpMV
 * (src/cuda.cu:143-146); without the division by 3, llgCPU's H4s (src/llgCPU.cpp:142-170). */
static void four_spin_add(const orc_ctx* c, const double* src, double* ch) {
    if (!c->q4ptr) return;
    for (uint32_t i = 0; i < c->n; i++) {
        double h[3] = {0.0, 0.0, 0.0};
        for (uint32_t q = c->q4ptr[i]; q < c->q4ptr[i + 1]; q++) {
            const double* sj = src + 3 * (size_t)c->q4j[q];
            const double* sk = src + 3 * (size_t)c->q4k[q];
            const double* sl = src + 3 * (size_t)c->q4l[q];
            const double skdotsl = sk[0] * sl[0] + sk[1] * sl[1] + sk[2] * sl[2];
            const double sjdotsl = sj[0] * sl[0] + sj[1] * sl[1] + sj[2] * sl[2];
            const double skdotsj = sk[0] * sj[0] + sk[1] * sj[1] + sk[2] * sj[2];
            for (int a = 0; a < 3; a++) {
                const double v = sj[a] * skdotsl + sk[a] * sjdotsl + sl[a] * skdotsj;
                h[a] -= c->q4div3 ? (c->q4jq * v) / 3.0 : c->q4jq * v;
            }
        }
        for (int a = 0; a < 3; a++) ch[3 * (size_t)i + a] += h[a];
    }
}

/* CH for a stage: (HDemag + exchange sum) (src/cufields.cu:201-203) or the FFT field, then the
 * four-spin term. */
static void stage_field(orc_ctx* c, const double* src, double* ch) {
    if (c->lr == ORC_LR_FFT) {
        longrange_field(c, src, ch);
        four_spin_add(c, src, ch);
        return;
    }
    for (uint32_t i = 0; i < c->n; i++) {
        double dot[3];
        exch_sum(c, src, i, dot);
        for (int a = 0; a < 3; a++) ch[3 * (size_t)i + a] = c->hdemag[3 * (size_t)i + a] + dot[a];
    }
    four_spin_add(c, src, ch);
}

int orc_set_four_spin(orc_ctx* c, const uint32_t* ptr, const uint32_t* j, const uint32_t* k, const uint32_t* l,
                      double jq, int div3) {
    freep(c->q4ptr); freep(c->q4j); freep(c->q4k); freep(c->q4l);
    c->q4ptr = c->q4j = c->q4k = c->q4l = NULL;
    if (!ptr) return 0;
    const uint32_t nq = ptr[c->n];
    c->q4ptr = (uint32_t*)malloc(sizeof(uint32_t) * (c->n + 1));
    c->q4j = (uint32_t*)malloc(sizeof(uint32_t) * (nq + 1));
    c->q4k = (uint32_t*)malloc(sizeof(uint32_t) * (nq + 1));
    c->q4l = (uint32_t*)malloc(sizeof(uint32_t) * (nq + 1));
    memcpy(c->q4ptr, ptr, sizeof(uint32_t) * (c->n + 1));
    memcpy(c->q4j, j, sizeof(uint32_t) * nq);
    memcpy(c->q4k, k, sizeof(uint32_t) * nq);
    memcpy(c->q4l, l, sizeof(uint32_t) * nq);
    c->q4jq = jq;
    c->q4div3 = div3;
    return 0;
}

int orc_field(orc_ctx* c, double* h) {
    if (c->lr == ORC_LR_DIPOLE) longrange_field(c, c->s, c->hdemag);
    stage_field(c, c->s, h);
    return 0;
}

static uint32_t replica_of(const orc_ctx* c, uint32_t i) {
    uint32_t lo = 0, hi = c->nrep;
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) / 2;
        if (c->rep_off[mid] <= i) lo = mid; else hi = mid;
    }
    return lo;
}

static void draw_noise(orc_ctx* c, uint64_t t) {
    const uint32_t n = c->n;
    if (c->noise_mode == ORC_NOISE_PHILOX) {
        for (uint32_t i = 0; i < n; i++) {
            uint32_t r = replica_of(c, i);
            orc_thermal_normals(c->seed, c->rep_stream[r], i - c->rep_off[r], t, c->noise + 3 * (size_t)i);
        }
    } else if (c->noise_mode == ORC_NOISE_MWC) {
        for (uint32_t i = 0; i < 3 * n; i++) c->noise[i] = orc_mwc_normal();
    } else {
        for (uint32_t i = 0; i < 3 * n; i++) {
            c->noise[i] = c->nbuf_len ? c->nbuf[c->nbuf_pos] : 0.0;
            if (c->nbuf_len) c->nbuf_pos = (c->nbuf_pos + 1) % c->nbuf_len;
        }
    }
}

/* Total field at spin i for stage spin s (anisotropy evaluated at s):
 * src/cuint.cu:66-137 (GPU order) or src/llgCPU.cpp:180-222 (CPU order).
 * lrn receives the thermal term. */
static void total_field(const orc_ctx* c, uint32_t i, const double* ch_exch, const double* s,
                        double h[3], double lrn[3]) {
    const uint32_t r = replica_of(c, i);
    const double TP = sqrt(c->rep_T[r]) * c->sigma[i];
    const double* xi = c->noise + 3 * (size_t)i;
    lrn[0] = xi[0] * TP; lrn[1] = xi[1] * TP; lrn[2] = xi[2] * TP;
    const double hs[3] = {c->cur_scale * c->hstag[3 * (size_t)i], c->cur_scale * c->hstag[3 * (size_t)i + 1],
                          c->cur_scale * c->hstag[3 * (size_t)i + 2]};
    if (c->flags & ORC_CPU_SUM_ORDER) {
        /* llgCPU: Hx holds the exchange only, HDemag and H4s are separate terms
         * (src/llgCPU.cpp:180). */
        const double* hx = ch_exch + 3 * (size_t)i;
        const double* hd = c->hdemag + 3 * (size_t)i;
        const double* h4 = c->h4s + 3 * (size_t)i;
        const double thz = (c->flags & ORC_CPU_THERMAL_Z_FROM_X) ? lrn[0] : lrn[2];
        h[0] = c->applied[0] + lrn[0] + hx[0] + hd[0] + h4[0] + hs[0];
        h[1] = c->applied[1] + lrn[1] + hx[1] + hd[1] + h4[1] + hs[1];
        h[2] = hx[2] + thz + c->applied[2] + hd[2] + h4[2] + hs[2];
        if (c->flags & ORC_CPU_THERMAL_Z_FROM_X) lrn[2] = thz;
    } else {
        const double* ch = ch_exch + 3 * (size_t)i;
        h[0] = ch[0] + hs[0] + lrn[0] + c->applied[0];
        h[1] = ch[1] + hs[1] + lrn[1] + c->applied[1];
        h[2] = ch[2] + hs[2] + lrn[2] + c->applied[2];
    }
    const double* d = c->k1udir + 3 * (size_t)i;
    const double k1u = c->k1u[i];
    const double sdn = s[0] * d[0] + s[1] * d[1] + s[2] * d[2];
    h[0] += (k1u * sdn * d[0]);
    h[1] += (k1u * sdn * d[1]);
    h[2] += (k1u * sdn * d[2]);
    const double sdk2perp = s[0] * c->k2perpdir[0] + s[1] * c->k2perpdir[1] + s[2] * c->k2perpdir[2];
    for (int a = 0; a < 3; a++) h[a] += (2.0 * c->k2perp / c->basemm) * sdk2perp * c->k2perpdir[a];
    const double sdk2par = s[0] * c->k2pardir[0] + s[1] * c->k2pardir[1] + s[2] * c->k2pardir[2];
    for (int a = 0; a < 3; a++) h[a] += (2.0 * c->k2par / c->basemm) * sdk2par * c->k2pardir[a];
    for (int dir = 0; dir < 3; dir++) {
        const double* pd = c->k4perpdirs + 3 * dir;
        const double* qd = c->k4pardirs + 3 * dir;
        const double sdk4perp = s[0] * pd[0] + s[1] * pd[1] + s[2] * pd[2];
        const double sdk4par = s[0] * qd[0] + s[1] * qd[1] + s[2] * qd[2];
        for (int a = 0; a < 3; a++) h[a] += (2.0 * c->k4perp / c->basemm) * sdk4perp * pd[a];
        for (int a = 0; a < 3; a++) h[a] += (2.0 * c->k4par / c->basemm) * sdk4par * qd[a];
    }
}

/* llgpf (S x H + lambda S x (S x H)), src/cuint.cu:142-150. scale multiplies llgpf first (rdt for RK). */
static void torque(double scale, double llgpf, double lambda, const double s[3], const double h[3], double f[3]) {
    const double sxh[3] = {s[1] * h[2] - s[2] * h[1], s[2] * h[0] - s[0] * h[2], s[0] * h[1] - s[1] * h[0]};
    const double sxsxh[3] = {s[1] * sxh[2] - s[2] * sxh[1], s[2] * sxh[0] - s[0] * sxh[2], s[0] * sxh[1] - s[1] * sxh[0]};
    for (int j = 0; j < 3; j++) {
        if (scale == 1.0) f[j] = llgpf * (sxh[j] + lambda * sxsxh[j]);
        else f[j] = scale * llgpf * (sxh[j] + lambda * sxsxh[j]);
    }
}

static void normalise(double v[3]) {
    const double mods = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    v[0] /= mods; v[1] /= mods; v[2] /= mods;
}

/* Site-field multiplier of step t: the ramp value, times the Gaussian envelope
 * amp exp(-x^2/2), x = (t dt - t0)/sigma, when a pulse is set (a driver calling
 * rampStag every step, src/cuda.cu:38-41). */
static void set_step_scale(orc_ctx* c, uint64_t t) {
    if (c->pulse_amp != 0.0) {
        const double x = ((double)t * c->dt - c->pulse_t0) / c->pulse_sigma;
        const double f = c->pulse_amp * exp(-0.5 * x * x);
        c->cur_scale = c->stag_scale * f;
    } else {
        c->cur_scale = c->stag_scale;
    }
}

int orc_set_pulse(orc_ctx* c, double amp, double t0, double sigma, double dt) {
    c->pulse_amp = amp; c->pulse_t0 = t0; c->pulse_sigma = sigma; c->dt = dt;
    return 0;
}

static void heun_step(orc_ctx* c, uint64_t t) {
    set_step_scale(c, t);
    const uint32_t n = c->n;
    double* hsave = NULL;
    if (c->lr == ORC_LR_DIPOLE && t % c->update == 0) {
        longrange_field(c, c->s, c->hdemag);
        if (c->flags & ORC_GPU_HDEMAG_FP32)
            for (size_t q = 0; q < 3 * (size_t)n; q++) c->hdemag[q] = (double)(float)c->hdemag[q];
    }
    if (c->flags & ORC_CPU_SUM_ORDER) {
        /* llgCPU: Hx = 0 + exchange sum; HDemag and H4s (recomputed from zero at each stage,
         * src/llgCPU.cpp:142-170,275-297) added as separate terms. */
        for (uint32_t i = 0; i < n; i++) {
            double dot[3];
            exch_sum(c, c->s, i, dot);
            for (int a = 0; a < 3; a++) c->h[3 * (size_t)i + a] = 0.0 + dot[a];
        }
        memset(c->h4s, 0, 3 * (size_t)n * sizeof(double));
        four_spin_add(c, c->s, c->h4s);
    } else {
        stage_field(c, c->s, c->h);
    }
    draw_noise(c, t);
    for (uint32_t i = 0; i < n; i++) {
        double h[3], lrn[3], f[3];
        const double* s = c->s + 3 * (size_t)i;
        total_field(c, i, c->h, s, h, lrn);
        torque(1.0, c->llgpf[i], c->lambda[i], s, h, f);
        double es[3];
        for (int j = 0; j < 3; j++) { c->fn[3 * (size_t)i + j] = f[j]; es[j] = s[j] + f[j] * c->rdt; }
        normalise(es);
        memcpy(c->es + 3 * (size_t)i, es, sizeof(es));
    }
    const int stale = (c->flags & ORC_GPU_CSR_DIP_STALE) && c->lr == ORC_LR_DIPOLE && c->exch == ORC_EXCH_CSR && !c->full;
    if (c->flags & ORC_CPU_SUM_ORDER) {
        for (uint32_t i = 0; i < n; i++) {
            double dot[3];
            exch_sum(c, c->es, i, dot);
            for (int a = 0; a < 3; a++) {
                if (c->flags & ORC_CPU_CORRECTOR_ACCUM) c->h[3 * (size_t)i + a] += dot[a];
                else c->h[3 * (size_t)i + a] = 0.0 + dot[a];
            }
        }
        memset(c->h4s, 0, 3 * (size_t)n * sizeof(double));
        four_spin_add(c, c->es, c->h4s);
    } else if (!stale) {
        if (c->flags & ORC_CPU_CORRECTOR_ACCUM) {
            hsave = dalloc(3 * (size_t)n);
            memcpy(hsave, c->h, 3 * (size_t)n * sizeof(double));
        }
        stage_field(c, c->es, c->h);
        if (hsave) {
            /* H(S') + exchange(S): the demag/long-range part is not accumulated. */
            for (uint32_t i = 0; i < n; i++)
                for (int a = 0; a < 3; a++)
                    c->h[3 * (size_t)i + a] += hsave[3 * (size_t)i + a] - c->hdemag[3 * (size_t)i + a];
            free(hsave);
        }
    }
    for (uint32_t i = 0; i < n; i++) {
        double h[3], lrn[3], f[3];
        const double* es = c->es + 3 * (size_t)i;
        total_field(c, i, c->h, es, h, lrn);
        torque(1.0, c->llgpf[i], c->lambda[i], es, h, f);
        double ps[3];
        for (int j = 0; j < 3; j++) ps[j] = c->s[3 * (size_t)i + j] + (0.5 * (c->fn[3 * (size_t)i + j] + f[j]) * c->rdt);
        normalise(ps);
        for (int j = 0; j < 3; j++) {
            c->s[3 * (size_t)i + j] = ps[j];
            c->det[3 * (size_t)i + j] = h[j] - lrn[j];
        }
    }
}

/* Cash-Karp tableau as used by src/cuintRK5.cu:44-54. */
static const double RK5_B21 = 0.2;
static const double RK5_B3[2] = {3.0 / 40.0, 9.0 / 40.0};
static const double RK5_B4[3] = {0.3, -0.9, 1.2};
static const double RK5_B5[4] = {-11.0 / 54, 2.5, -70.0 / 27.0, 35.0 / 27.0};
static const double RK5_B6[5] = {1631.0 / 55296.0, 175.0 / 512.0, 575.0 / 13824.0, 44275.0 / 110592.0, 253.0 / 4096.0};
static const double RK5_C[6] = {37.0 / 378.0, 0.0, 250.0 / 621.0, 125.0 / 594.0, 0.0, 512.0 / 1771.0};

/* One RK4 / RK5 step with the launch sequence of src/cudaRK4.cu:38-233 and
 * src/cudaRK5.cu (SpMV of the stage spin, then the stage kernel). */
static void rk_step(orc_ctx* c, uint64_t t) {
    set_step_scale(c, t);
    const uint32_t n = c->n;
    const int nst = c->integrator == ORC_RK4 ? 4 : 6;
    const int dbl = (c->flags & ORC_RK_DOUBLE_RDT) != 0;
    const int mixed = (c->flags & ORC_RK_STAGE_SPIN_MIXED) != 0;
    draw_noise(c, t);
    if (c->lr == ORC_LR_DIPOLE && t % c->update == 0) {
        longrange_field(c, c->s, c->hdemag);
        if (c->flags & ORC_GPU_HDEMAG_FP32)
            for (size_t q = 0; q < 3 * (size_t)n; q++) c->hdemag[q] = (double)(float)c->hdemag[q];
    }
    for (int st = 0; st < nst; st++) {
        stage_field(c, st == 0 ? c->s : c->es, c->h);
        for (uint32_t i = 0; i < n; i++) {
            const double* S = c->s + 3 * (size_t)i;
            double sv[3];
            if (st == 0) memcpy(sv, S, sizeof(sv));
            else if (mixed) { sv[0] = c->es[3 * (size_t)i]; sv[1] = S[1]; sv[2] = c->es[3 * (size_t)i + 2]; }
            else memcpy(sv, c->es + 3 * (size_t)i, sizeof(sv));
            double h[3], lrn[3], k[3];
            total_field(c, i, c->h, sv, h, lrn);
            torque(c->rdt, c->llgpf[i], c->lambda[i], sv, h, k);
            memcpy(c->k[st] + 3 * (size_t)i, k, sizeof(k));
            if (st == nst - 1) continue;
            double es[3];
            for (int j = 0; j < 3; j++) {
                double inc;
                if (nst == 4) {
                    const double a = st == 2 ? 1.0 : 0.5;
                    if (dbl) inc = st == 2 ? c->rdt * k[j] : c->rdt * k[j] * 0.5;
                    else inc = k[j] * a;
                } else {
                    double sum;
                    const size_t q = 3 * (size_t)i + j;
                    if (st == 0) sum = RK5_B21 * k[j];
                    else if (st == 1) sum = RK5_B3[0] * c->k[0][q] + RK5_B3[1] * k[j];
                    else if (st == 2) sum = RK5_B4[0] * c->k[0][q] + RK5_B4[1] * c->k[1][q] + RK5_B4[2] * k[j];
                    else if (st == 3)
                        sum = RK5_B5[0] * c->k[0][q] + RK5_B5[1] * c->k[1][q] + RK5_B5[2] * c->k[2][q] + RK5_B5[3] * k[j];
                    else
                        sum = RK5_B6[0] * c->k[0][q] + RK5_B6[1] * c->k[1][q] + RK5_B6[2] * c->k[2][q] +
                              RK5_B6[3] * c->k[3][q] + RK5_B6[4] * k[j];
                    inc = dbl ? c->rdt * sum : sum;
                }
                es[j] = S[j] + inc;
            }
            normalise(es);
            memcpy(c->es + 3 * (size_t)i, es, sizeof(es));
        }
    }
    for (uint32_t i = 0; i < n; i++) {
        double ls[3];
        for (int j = 0; j < 3; j++) {
            const size_t q = 3 * (size_t)i + j;
            if (nst == 4)
                ls[j] = c->s[q] + c->k[0][q] * (1.0 / 6.0) + c->k[1][q] * (1.0 / 3.0) + c->k[2][q] * (1.0 / 3.0) +
                        c->k[3][q] * (1.0 / 6.0);
            else
                ls[j] = c->s[q] + c->k[0][q] * RK5_C[0] + c->k[1][q] * RK5_C[1] + c->k[2][q] * RK5_C[2] +
                        c->k[3][q] * RK5_C[3] + c->k[4][q] * RK5_C[4] + c->k[5][q] * RK5_C[5];
        }
        normalise(ls);
        memcpy(c->s + 3 * (size_t)i, ls, sizeof(ls));
    }
}

int orc_run(orc_ctx* c, uint64_t t0, uint64_t nsteps) {
    for (uint64_t t = t0; t < t0 + nsteps; t++) {
        if (c->integrator == ORC_HEUN) heun_step(c, t);
        else rk_step(c, t);
    }
    return 0;
}

int orc_magnetisation(const orc_ctx* c, uint32_t nsub, const uint32_t* sublattice, double* out) {
    for (uint32_t r = 0; r < c->nrep; r++) {
        double* m = out + (size_t)r * nsub * 3;
        uint32_t* cnt = (uint32_t*)calloc(nsub, sizeof(uint32_t));
        for (uint32_t q = 0; q < 3 * nsub; q++) m[q] = 0.0;
        for (uint32_t i = c->rep_off[r]; i < c->rep_off[r + 1]; i++) {
            const uint32_t sl = sublattice ? sublattice[i] : 0;
            for (int a = 0; a < 3; a++) m[3 * sl + a] += c->s[3 * (size_t)i + a];
            cnt[sl]++;
        }
        for (uint32_t sl = 0; sl < nsub; sl++) {
            const double oones = 1. / (double)(cnt[sl] ? cnt[sl] : 1);
            for (int a = 0; a < 3; a++) m[3 * sl + a] *= oones;
        }
        free(cnt);
    }
    return 0;
}

/* ------------------------------------------------------------------ */
int orc_csr_to_dia(uint32_t n, const uint32_t* xadj, const uint32_t* adjncy, const double* val9,
                   int32_t* offsets, double* data9) {
    /* checkdiag as filled in src/exch_unitcell.cpp:374-391 */
    uint32_t* check = (uint32_t*)calloc(2 * (size_t)n, sizeof(uint32_t));
    for (uint32_t i = 0; i < n; i++)
        for (uint32_t k = xadj[i]; k < xadj[i + 1]; k++) check[(int64_t)n + (int64_t)adjncy[k] - (int64_t)i]++;
    int count = 0;
    for (uint32_t q = 0; q + 1 < 2 * n; q++) {
        if (check[q] > 0) {
            if (offsets) offsets[count] = (int32_t)q - (int32_t)n;
            count++;
        }
    }
    free(check);
    if (!offsets) return count;
    const size_t m = (size_t)count * n;
    memset(data9, 0, 9 * m * sizeof(double));
    for (int d = 0; d < count; d++) {
        const int32_t diag = offsets[d];
        const int32_t num_elem = diag <= 0 ? diag + (int32_t)n : (int32_t)n - diag;
        int32_t row = diag <= 0 ? -diag : 0, col = diag <= 0 ? 0 : diag;
        for (int32_t e = 0; e < num_elem; e++, row++, col++) {
            for (uint32_t k = xadj[row]; k < xadj[row + 1]; k++) {
                if (adjncy[k] == (uint32_t)col) {
                    for (int q = 0; q < 9; q++) data9[(size_t)q * m + (size_t)d * n + row] = val9[9 * (size_t)k + q];
                }
            }
        }
    }
    return count;
}

int orc_build_dipole_nr(const uint32_t* dim, const uint32_t* nk, const double* abc, double muB,
                        double mu_scale, double* nr) {
    uint32_t L[3], M[3];
    int mono[3];
    for (int l = 0; l < 3; l++) { L[l] = dim[l] * nk[l]; M[l] = 2 * dim[l] * nk[l]; mono[l] = L[l] < 2; }
    const size_t p = (size_t)M[0] * M[1] * M[2];
    const int I[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    for (uint32_t i = 0; i < M[0]; i++)
        for (uint32_t j = 0; j < M[1]; j++)
            for (uint32_t k = 0; k < M[2]; k++) {
                if (i == 0 && j == 0 && k == 0) continue;
                int lc[3] = {(int)i, (int)j, (int)k}, tc[3] = {(int)i, (int)j, (int)k};
                if ((tc[0] > 0 && mono[0]) || (tc[1] > 0 && mono[1]) || (tc[2] > 0 && mono[2])) continue;
                double rij[3];
                for (int l = 0; l < 3; l++) {
                    if ((uint32_t)lc[l] > L[l]) { lc[l] = (int)L[l] - lc[l]; tc[l] = (int)M[l] + lc[l]; }
                    rij[l] = (double)lc[l] * abc[l] / (double)nk[l];
                }
                const double mrij = sqrt(rij[0] * rij[0] + rij[1] * rij[1] + rij[2] * rij[2]);
                const double oomrij3 = 1. / (mrij * mrij * mrij);
                const double eij[3] = {rij[0] / mrij, rij[1] / mrij, rij[2] / mrij};
                const size_t cell = ((size_t)tc[0] * M[1] + tc[1]) * M[2] + tc[2];
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 3; b++)
                        nr[(size_t)(3 * a + b) * p + cell] += 1e-7 * ((3.0 * eij[a] * eij[b]) - I[a][b]) * oomrij3 * mu_scale * muB;
            }
    return 0;
}

int orc_fold_exchange_nr(const uint32_t* mesh, uint32_t nshell, const int32_t* shell_vec,
                         const double* J9, double mu_muB, double* nr) {
    const size_t p = (size_t)mesh[0] * mesh[1] * mesh[2];
    unsigned char* check = (unsigned char*)calloc(p, 1);
    int total = 0;
    for (uint32_t sh = 0; sh < nshell; sh++) {
        const int32_t* lc = shell_vec + 3 * sh;
        const double* J = J9 + 9 * sh;
        for (int wrap = 0; wrap < 3; wrap++) {
            int rc[3] = {lc[wrap % 3], lc[(1 + wrap) % 3], lc[(2 + wrap) % 3]};
            for (int swap = 0; swap < 2; swap++) {
                if (swap == 1) { int t = rc[1]; rc[1] = rc[2]; rc[2] = t; }
                for (int a = 0; a < 2; a++)
                    for (int b = 0; b < 2; b++)
                        for (int cc = 0; cc < 2; cc++) {
                            int wc[3] = {a ? rc[0] : -rc[0], b ? rc[1] : -rc[1], cc ? rc[2] : -rc[2]};
                            for (int x = 0; x < 3; x++) if (wc[x] < 0) wc[x] += (int)mesh[x];
                            const size_t cell = ((size_t)wc[0] * mesh[1] + wc[1]) * mesh[2] + wc[2];
                            if (check[cell]) continue;
                            for (int al = 0; al < 3; al++) nr[(size_t)(4 * al) * p + cell] += J[4 * al] / mu_muB;
                            const int od[6] = {1, 2, 3, 5, 6, 7};
                            for (int q = 0; q < 6; q++) nr[(size_t)od[q] * p + cell] += J[od[q]] / mu_muB;
                            check[cell] = 1;
                            total++;
                        }
            }
        }
    }
    free(check);
    return total;
}
