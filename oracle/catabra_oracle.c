/*
 * catabra_oracle.c -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
 *
 * CPU restatement of CatabraFFT.jl's 1D complex-to-complex FFT, used only as
 * the checker in tests/, in __graft_entry__.smoke() and as the timed CPU
 * baseline in bench.py.  Nothing in the shipped library links or calls it.
 *
 * It follows the reference algorithm step by step (paths relative to the
 * CatabraFFT.jl project):
 *   - strategy choice             src/kernel.jl:72-92  (generate_and_cache_fft!)
 *   - pure radix families         src/kernel.jl:119-143, src/radix_plan.jl:100-138
 *   - pass -> codelet mapping     src/radix_exec.jl:49-70, :105-113
 *   - codelets                    src/radix_2_codelets.jl, radix_3_codelets.jl,
 *                                 radix_5_codelets.jl, radix_7_codelets.jl
 *   - factor heuristic            src/kernel.jl:146-191 (find_closest_factors)
 *   - mixed radix (four-step)     src/mixed_radix.jl:30-78
 *   - Rader                       src/prime.jl:5-81
 *   - fft / ifft / bfft           src/CatabraFFT.jl:65-115
 *
 * Parity status: the reference is Julia and Julia is absent on every machine
 * of this build, so this restatement cannot be diffed against outputs of the
 * reference itself.  It is pinned instead against the reference's own test
 * contract (test/runtests.jl compares CatabraFFT.fft with FFTW.fft): the test
 * suite checks it against numpy's pocketfft and an mpmath direct DFT on every
 * size class the reference tests.  Parity with the reference's *outputs* is
 * therefore "unpinned" in the strict sense.
 *
 * Deliberate, documented deviations (all found by reading the reference):
 *   1. Rader twiddle clobber (prime.jl:61 passes its captured W as the input
 *      of F, and pure-radix F with >=3 passes uses its input as ping-pong
 *      scratch).  Mode ORACLE_RADER_FIXED (default) copies W first, which is
 *      what the reference computes on the first call in a fresh process;
 *      mode ORACLE_RADER_FAITHFUL keeps the clobbering behaviour.
 *   2. Layered radix-2/3/4 codelets are not Stockham-correct for n1 > 1
 *      (radix_2_codelets.jl:530-570,608-640; radix_3_codelets.jl:276-336).
 *      Default plans never use them as layered passes; this file implements
 *      the correct Stockham pass for them (reachable only by explicit plans).
 *   3. fft!(x) calls fft_kernel!(x, x) (CatabraFFT.jl:46-49) with aliased
 *      in/out buffers, which breaks every multi-pass Stockham plan.  The
 *      in-place entry here computes the intended transform.
 *
 * Build: oracle/Makefile builds liboracle_f64.so (double) and
 * liboracle_f32.so (-DORACLE_F32: the reference's ComplexF32 arithmetic).
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifdef ORACLE_F32
#define REAL float
#define PFX(name) co32_##name
#else
#define REAL double
#define PFX(name) co64_##name
#endif

typedef struct { REAL re, im; } cx;

/* ---- complex arithmetic in Julia Base's evaluation order (no FMA) ---- */
static inline cx C(REAL r, REAL i) { cx z; z.re = r; z.im = i; return z; }
static inline cx add(cx a, cx b) { return C(a.re + b.re, a.im + b.im); }
static inline cx sub(cx a, cx b) { return C(a.re - b.re, a.im - b.im); }
/* Julia: Complex(re(z)re(w) - im(z)im(w), re(z)im(w) + im(z)re(w)) */
static inline cx mul(cx a, cx b) {
    return C(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
static inline cx rmul(REAL s, cx a) { return C(s * a.re, s * a.im); }
static inline cx neg_i(cx a) { return C(a.im, -a.re); }      /* -im * a */
static inline cx pos_i(cx a) { return C(-a.im, a.re); }      /*  im * a */
static inline cx conjc(cx a) { return C(a.re, -a.im); }

/* ---- cispi with careful argument reduction (Julia's sincospi is <1ulp) ---- */
static void sincospi_ld(double x, double *s, double *c) {
    const long double PI_L = 3.141592653589793238462643383279502884L;
    double ax = fabs(x);
    double t = fmod(ax, 2.0);              /* exact */
    double ssign = 1.0, csign = 1.0;
    if (t >= 1.0) { t -= 1.0; ssign = -ssign; csign = -csign; }
    if (t > 0.5) { t = 1.0 - t; csign = -csign; }
    int swap = 0;
    if (t > 0.25) { t = 0.5 - t; swap = 1; }
    long double a = PI_L * (long double)t;
    double sv = (double)sinl(a), cv = (double)cosl(a);
    if (swap) { double tmp = sv; sv = cv; cv = tmp; }
    sv *= ssign; cv *= csign;
    if (x < 0) sv = -sv;
    *s = sv; *c = cv;
}
static inline cx cispi_T(REAL x) {           /* cispi evaluated in type T */
    double s, c;
    sincospi_ld((double)x, &s, &c);
    return C((REAL)c, (REAL)s);
}
static inline cx cispi_f64(double x) {       /* cispi evaluated in Float64 */
    double s, c;
    sincospi_ld(x, &s, &c);
    return C((REAL)c, (REAL)s);
}

/* ---- codelet constants (radix_2_codelets.jl:4-6, radix_3_codelets.jl:3-8,
 *      radix_5_codelets.jl:3-4, radix_7_codelets.jl:3-5), converted to T ---- */
#define INV_SQRT2 ((REAL)0.7071067811865475)
#define CP_3_8 ((REAL)0.3826834323650898)
#define SP_3_8 ((REAL)0.9238795325112867)
#define R3_CP ((REAL)0.5)
#define R3_SP ((REAL)0.8660254037844386)
#define CP_2_9 ((REAL)0.766044443118978)
#define SP_2_9 ((REAL)0.6427876096865393)
#define CP_4_9 ((REAL)0.17364817766693041)
#define SP_4_9 ((REAL)0.984807753012208)
#define CP_8_9 ((REAL)0.9396926207859083)
#define SP_8_9 ((REAL)0.3420201433256689)
#define R5_CP1 ((REAL)0.8090169943749473)
#define R5_SP1 ((REAL)0.5877852522924731)
#define R5_CP2 ((REAL)0.30901699437494734)
#define R5_SP2 ((REAL)0.9510565162951536)
#define R7_CP1 ((REAL)0.6234898018587336)
#define R7_SP1 ((REAL)0.7818314824680298)
#define R7_CP2 ((REAL)0.22252093395631448)
#define R7_SP2 ((REAL)0.9749279121818236)
#define R7_CP3 ((REAL)0.9009688679024191)
#define R7_SP3 ((REAL)0.4338837391175581)

/* ---- DFT_r butterflies: a[0..r-1] -> o[0..r-1], un-twiddled ----
 * Each mirrors the expression tree of the reference codelet body. */
static void bfly2(const cx *a, cx *o) {            /* radix_2_codelets.jl:654-657 */
    o[0] = add(a[0], a[1]); o[1] = sub(a[0], a[1]);
}
static void bfly4(const cx *a, cx *o) {            /* radix_2_codelets.jl:574-579 */
    cx t1 = add(a[0], a[2]), t2 = sub(a[0], a[2]);
    cx t3 = add(a[1], a[3]), t4 = neg_i(sub(a[1], a[3]));
    o[0] = add(t1, t3); o[1] = add(t2, t4); o[2] = sub(t1, t3); o[3] = sub(t2, t4);
}
static void bfly8(const cx *a, cx *o) {            /* radix_2_codelets.jl:486-501 */
    const cx Q4 = C(INV_SQRT2, -INV_SQRT2);        /* INV_SQRT2 * (1 - im)  */
    const cx Q3 = C(-INV_SQRT2, -INV_SQRT2);       /* INV_SQRT2 * (-1 - im) */
    cx t13 = add(a[0], a[4]), t14 = sub(a[0], a[4]);
    cx t15 = add(a[2], a[6]), t16 = neg_i(sub(a[2], a[6]));
    cx t5 = add(t13, t15), t6 = add(t14, t16);
    cx t7 = sub(t13, t15), t8 = sub(t14, t16);
    cx t17 = add(a[1], a[5]), t18 = sub(a[1], a[5]);
    cx t19 = add(a[3], a[7]), t20 = neg_i(sub(a[3], a[7]));
    cx t9 = add(t17, t19), t10 = mul(Q4, add(t18, t20));
    cx t11 = neg_i(sub(t17, t19)), t12 = mul(Q3, sub(t18, t20));
    o[0] = add(t5, t9); o[1] = add(t6, t10); o[2] = add(t7, t11); o[3] = add(t8, t12);
    o[4] = sub(t5, t9); o[5] = sub(t6, t10); o[6] = sub(t7, t11); o[7] = sub(t8, t12);
}
static void bfly16(const cx *x, cx *o) {           /* radix_2_codelets.jl:87-119 */
    const cx Q4 = C(INV_SQRT2, -INV_SQRT2), Q3 = C(-INV_SQRT2, -INV_SQRT2);
    const cx A = C(SP_3_8, -CP_3_8), B = C(CP_3_8, -SP_3_8);
    const cx Cc = C(-CP_3_8, -SP_3_8), D = C(-SP_3_8, -CP_3_8);
    cx t45 = add(x[0], x[8]), t46 = sub(x[0], x[8]);
    cx t47 = add(x[4], x[12]), t48 = neg_i(sub(x[4], x[12]));
    cx t37 = add(t45, t47), t38 = add(t46, t48), t39 = sub(t45, t47), t40 = sub(t46, t48);
    cx t49 = add(x[2], x[10]), t50 = sub(x[2], x[10]);
    cx t51 = add(x[6], x[14]), t52 = neg_i(sub(x[6], x[14]));
    cx t41 = add(t49, t51), t42 = mul(Q4, add(t50, t52));
    cx t43 = neg_i(sub(t49, t51)), t44 = mul(Q3, sub(t50, t52));
    cx t21 = add(t37, t41), t22 = add(t38, t42), t23 = add(t39, t43), t24 = add(t40, t44);
    cx t25 = sub(t37, t41), t26 = sub(t38, t42), t27 = sub(t39, t43), t28 = sub(t40, t44);
    cx t61 = add(x[1], x[9]), t62 = sub(x[1], x[9]);
    cx t63 = add(x[5], x[13]), t64 = neg_i(sub(x[5], x[13]));
    cx t53 = add(t61, t63), t54 = add(t62, t64), t55 = sub(t61, t63), t56 = sub(t62, t64);
    cx t65 = add(x[3], x[11]), t66 = sub(x[3], x[11]);
    cx t67 = add(x[7], x[15]), t68 = neg_i(sub(x[7], x[15]));
    cx t57 = add(t65, t67), t58 = mul(Q4, add(t66, t68));
    cx t59 = neg_i(sub(t65, t67)), t60 = mul(Q3, sub(t66, t68));
    cx t29 = add(t53, t57), t30 = mul(A, add(t54, t58));
    cx t31 = mul(Q4, add(t55, t59)), t32 = mul(B, add(t56, t60));
    cx t33 = neg_i(sub(t53, t57)), t34 = mul(Cc, sub(t54, t58));
    cx t35 = mul(Q3, sub(t55, t59)), t36 = mul(D, sub(t56, t60));
    o[0] = add(t21, t29); o[1] = add(t22, t30); o[2] = add(t23, t31); o[3] = add(t24, t32);
    o[4] = add(t25, t33); o[5] = add(t26, t34); o[6] = add(t27, t35); o[7] = add(t28, t36);
    o[8] = sub(t21, t29); o[9] = sub(t22, t30); o[10] = sub(t23, t31); o[11] = sub(t24, t32);
    o[12] = sub(t25, t33); o[13] = sub(t26, t34); o[14] = sub(t27, t35); o[15] = sub(t28, t36);
}
static void bfly3(const cx *x, cx *o) {            /* radix_3_codelets.jl:382-390 */
    cx a = x[0], b = x[1], c = x[2];
    cx bpc = add(b, c);
    cx jbmcS = rmul(R3_SP, pos_i(sub(b, c)));      /* (im*(b - c))*Sp */
    cx ambpcCp = sub(a, rmul(R3_CP, bpc));
    o[0] = add(a, bpc); o[1] = sub(ambpcCp, jbmcS); o[2] = add(ambpcCp, jbmcS);
}
static void bfly9(const cx *x, cx *o) {            /* radix_3_codelets.jl:18-37 */
    cx a = x[0], b = x[1], c = x[2], d = x[3], e = x[4], f = x[5], g = x[6], h = x[7], i = x[8];
    cx t1 = add(b, i), t2 = add(c, h), t3 = add(d, g), t4 = add(e, f);
    cx m1 = sub(i, b), m2 = sub(h, c), m3 = sub(g, d), m4 = sub(f, e);
    cx t3_Cp = rmul(R3_CP, t3), m3_Sp = rmul(R3_SP, m3);
    cx t11 = add(add(t1, t2), t4), t12 = add(a, t3);
    cx x1 = sub(sub(add(add(a, rmul(CP_2_9, t1)), rmul(CP_4_9, t2)), t3_Cp), rmul(CP_8_9, t4));
    cx y1 = pos_i(add(add(add(rmul(SP_2_9, m1), rmul(SP_4_9, m2)), m3_Sp), rmul(SP_8_9, m4)));
    cx x2 = add(sub(sub(add(a, rmul(CP_4_9, t1)), rmul(CP_8_9, t2)), t3_Cp), rmul(CP_2_9, t4));
    cx y2 = pos_i(sub(sub(add(rmul(SP_4_9, m1), rmul(SP_8_9, m2)), m3_Sp), rmul(SP_2_9, m4)));
    cx x3 = add(rmul(-R3_CP, t11), t12);
    cx y3 = rmul(R3_SP, pos_i(add(sub(m1, m2), m4)));   /* value of im*Sp*(m1-m2+m4) */
    cx x4 = add(sub(add(sub(a, rmul(CP_8_9, t1)), rmul(CP_2_9, t2)), t3_Cp), rmul(CP_4_9, t4));
    cx y4 = pos_i(sub(add(sub(rmul(SP_8_9, m1), rmul(SP_2_9, m2)), m3_Sp), rmul(SP_4_9, m4)));
    o[0] = add(t11, t12); o[1] = add(x1, y1); o[2] = add(x2, y2); o[3] = add(x3, y3);
    o[4] = add(x4, y4); o[5] = sub(x4, y4); o[6] = sub(x3, y3); o[7] = sub(x2, y2); o[8] = sub(x1, y1);
}
static void bfly5(const cx *x, cx *o) {            /* radix_5_codelets.jl:12-23 */
    cx a = x[0], b = x[1], c = x[2], d = x[3], e = x[4];
    cx bpe = add(b, e), dpc = add(d, c), bme = sub(b, e), dmc = sub(d, c);
    cx x1 = sub(add(a, rmul(R5_CP2, bpe)), rmul(R5_CP1, dpc));
    cx y1 = pos_i(add(rmul(-R5_SP2, bme), rmul(R5_SP1, dmc)));
    cx x2 = add(sub(a, rmul(R5_CP1, bpe)), rmul(R5_CP2, dpc));
    cx y2 = pos_i(add(rmul(R5_SP1, bme), rmul(R5_SP2, dmc)));
    o[0] = add(add(a, bpe), dpc); o[1] = add(x1, y1); o[2] = sub(x2, y2);
    o[3] = add(x2, y2); o[4] = sub(x1, y1);
}
static void bfly7(const cx *x, cx *o) {            /* radix_7_codelets.jl:11-25 */
    cx a = x[0], b = x[1], c = x[2], d = x[3], e = x[4], f = x[5], g = x[6];
    cx bpg = add(b, g), cpf = add(c, f), dpe = add(d, e);
    cx bmg = sub(b, g), cmf = sub(c, f), dme = sub(d, e);
    cx x1 = sub(sub(add(a, rmul(R7_CP1, bpg)), rmul(R7_CP2, cpf)), rmul(R7_CP3, dpe));
    cx y1 = pos_i(sub(sub(rmul(-R7_SP1, bmg), rmul(R7_SP2, cmf)), rmul(R7_SP3, dme)));
    cx x2 = add(sub(sub(a, rmul(R7_CP2, bpg)), rmul(R7_CP3, cpf)), rmul(R7_CP1, dpe));
    cx y2 = pos_i(add(add(rmul(-R7_SP2, bmg), rmul(R7_SP3, cmf)), rmul(R7_SP1, dme)));
    cx x3 = sub(add(sub(a, rmul(R7_CP3, bpg)), rmul(R7_CP1, cpf)), rmul(R7_CP2, dpe));
    cx y3 = pos_i(sub(add(rmul(-R7_SP3, bmg), rmul(R7_SP1, cmf)), rmul(R7_SP2, dme)));
    o[0] = add(add(add(a, bpg), cpf), dpe); o[1] = add(x1, y1); o[2] = add(x2, y2);
    o[3] = add(x3, y3); o[4] = sub(x3, y3); o[5] = sub(x2, y2); o[6] = sub(x1, y1);
}

static void bfly(int r, const cx *a, cx *o) {
    switch (r) {
    case 2: bfly2(a, o); break;   case 3: bfly3(a, o); break;
    case 4: bfly4(a, o); break;   case 5: bfly5(a, o); break;
    case 7: bfly7(a, o); break;   case 8: bfly8(a, o); break;
    case 9: bfly9(a, o); break;   case 16: bfly16(a, o); break;
    default: abort();
    }
}

/* Twiddle power chains w[1..r-1] from w1, exactly as each codelet builds them
 * (radix_2_codelets.jl:14-28,423-429,548-550; radix_3_codelets.jl:180-187,
 *  radix_5_codelets.jl:89-92; radix_7_codelets.jl:106-111). */
static void twiddle_chain(int r, cx w1, cx *w) {
    w[1] = w1;
    switch (r) {
    case 2: break;
    case 3: w[2] = mul(w1, w1); break;
    case 4: w[2] = mul(w1, w1); w[3] = mul(w[2], w1); break;
    case 5: w[2] = mul(w1, w1); w[3] = mul(w[2], w1); w[4] = mul(w[3], w1); break;
    case 7: for (int j = 2; j < 7; j++) w[j] = mul(w[j - 1], w1); break;
    case 8:
        w[2] = mul(w1, w1); w[3] = mul(w1, w[2]); w[4] = mul(w[2], w[2]);
        w[5] = mul(w[2], w[3]); w[6] = mul(w[3], w[3]); w[7] = mul(w[3], w[4]); break;
    case 9:
        w[2] = mul(w1, w1); w[3] = mul(w[2], w1); w[4] = mul(w[2], w[2]); w[5] = mul(w[3], w[2]);
        w[6] = mul(w[3], w[3]); w[7] = mul(w[4], w[3]); w[8] = mul(w[4], w[4]); break;
    case 16:
        w[2] = mul(w1, w1); w[3] = mul(w1, w[2]); w[4] = mul(w[2], w[2]); w[5] = mul(w1, w[4]);
        w[6] = mul(w[2], w[4]); w[7] = mul(w[3], w[4]); w[8] = mul(w[4], w[4]);
        w[9] = mul(w[5], w[4]); w[10] = mul(w[5], w[5]); w[11] = mul(w[5], w[6]);
        w[12] = mul(w[6], w[6]); w[13] = mul(w[6], w[7]); w[14] = mul(w[8], w[6]);
        w[15] = mul(w[7], w[8]); break;
    default: abort();
    }
}

/* fft{r}_shell_layered!(y, x, s, n1, theta): one Stockham pass (0-based):
 *   a_k = x[q + s(p + k n1)],  y[q + s(r p + j)] = w_j(p) * DFT_r(a)_j
 * with w_1(p) = cispi(T(-p*theta)) and higher powers by the chain above. */
static void shell_layered(int r, cx *y, const cx *x, int64_t s, int64_t n1, double theta) {
    cx a[16], o[16], w[16];
    for (int64_t p = 0; p < n1; p++) {
        cx w1 = (r == 16) ? cispi_f64(-(double)p * theta)   /* radix 16 uses Float64 cispi */
                          : cispi_T((REAL)(-(double)p * theta));
        if (p > 0) twiddle_chain(r, w1, w);
        for (int64_t q = 0; q < s; q++) {
            for (int k = 0; k < r; k++) a[k] = x[q + s * (p + k * n1)];
            bfly(r, a, o);
            y[q + s * (r * p)] = o[0];
            for (int j = 1; j < r; j++)
                y[q + s * (r * p + j)] = (p > 0) ? mul(w[j], o[j]) : o[j];
        }
    }
}
/* fft{r}_shell!(y, x, s) / fft{r}_shell_y!(y, s): last, un-twiddled pass. */
static void shell_last(int r, cx *y, const cx *x, int64_t s) {
    cx a[16], o[16];
    for (int64_t q = 0; q < s; q++) {
        for (int k = 0; k < r; k++) a[k] = x[q + s * k];
        bfly(r, a, o);
        for (int j = 0; j < r; j++) y[q + s * j] = o[j];
    }
}

/* ---------------------------- plan tree ---------------------------------- */
enum { K_COPY = 0, K_RADIX = 1, K_MIXED = 2, K_RADER = 3 };
#define MAXPASS 64
typedef struct node {
    int kind;
    int64_t n;
    int npass;
    int radix[MAXPASS];
    /* mixed radix */
    int64_t p, m;
    cx *W;                 /* (m-1) x (p-1), column i-1 holds w^i */
    struct node *Fp, *Fm;
    /* rader */
    int64_t gen;
    int64_t *gen_seq, *inv_seq;
    cx *Wr, *Wr_work;      /* Wr: pristine twiddles; Wr_work: the buffer handed to F */
    struct node *F;
    struct node *next;     /* cache chain */
} node;

static node *g_cache = NULL;
static int g_rader_mode = 0;   /* 0 = fixed (copy W), 1 = faithful (W clobbered) */

static int is_power_of(int64_t n, int64_t p) {     /* kernel.jl:102-110 */
    while (n > 1) { if (n % p != 0) return 0; n /= p; }
    return 1;
}
static int isprime64(int64_t n) {
    if (n < 2) return 0;
    if (n % 2 == 0) return n == 2;
    for (int64_t d = 3; d * d <= n; d += 2) if (n % d == 0) return 0;
    return 1;
}
static int64_t isqrt64(int64_t n) {
    int64_t r = (int64_t)sqrt((double)n);
    while (r * r > n) r--;
    while ((r + 1) * (r + 1) <= n) r++;
    return r;
}
static int64_t powmod64(int64_t b, int64_t e, int64_t m) {
    __int128 r = 1, x = b % m;
    while (e > 0) { if (e & 1) r = (r * x) % m; x = (x * x) % m; e >>= 1; }
    return (int64_t)r;
}

/* create_std_radix_plan (radix_plan.jl:100-138): greedy, largest radix first */
static int std_radix_plan(int64_t n, const int *radices, int nr, int *out) {
    int np = 0;
    int64_t rem = n;
    while (rem > 1) {
        int chosen = 0;
        for (int i = 0; i < nr; i++) if (rem % radices[i] == 0) { chosen = radices[i]; break; }
        if (!chosen || np >= MAXPASS) return -1;
        out[np++] = chosen;
        rem /= chosen;
    }
    return np;
}

/* find_closest_factors (kernel.jl:169-191) with prime-power preference */
static void find_closest_factors(int64_t n, int64_t *p_out, int64_t *m_out) {
    if (isprime64(n)) { *p_out = 1; *m_out = n; return; }
    /* return_sorted_prime_powers (kernel.jl:146-164), descending */
    int64_t pw[256]; int npw = 0;
    const int64_t primes[4] = {2, 3, 5, 7};
    for (int i = 0; i < 4; i++) {
        int64_t v = primes[i];
        while (v <= n && npw < 256) { pw[npw++] = v; if (v > INT64_MAX / primes[i]) break; v *= primes[i]; }
    }
    for (int i = 0; i < npw; i++)
        for (int j = i + 1; j < npw; j++)
            if (pw[j] > pw[i]) { int64_t t = pw[i]; pw[i] = pw[j]; pw[j] = t; }
    for (int i = 0; i < npw; i++)
        if (n % pw[i] == 0) { *p_out = pw[i]; *m_out = n / pw[i]; return; }
    int64_t p = isqrt64(n);
    while (n % p != 0) { p -= 1; if (p == 1) { *p_out = 1; *m_out = n; return; } }
    *p_out = p; *m_out = n / p;
}

static node *get_plan(int64_t n);

/* D(p, m, T) (mixed_radix.jl:30-41) */
static cx *make_D(int64_t p, int64_t m) {
    int64_t n = p * m;
    cx *d = (cx *)calloc((size_t)((p - 1) * (m - 1) + 1), sizeof(cx));
    REAL unit = (REAL)(-2.0 / (double)n);              /* T(-2/(p*m)) */
    for (int64_t k = 1; k <= m - 1; k++) d[k - 1] = cispi_T(unit * (REAL)k);
    for (int64_t j = 2; j <= p - 1; j++)
        for (int64_t k = 0; k < m - 1; k++)
            d[(j - 1) * (m - 1) + k] = mul(d[k], d[(j - 2) * (m - 1) + k]);
    return d;
}

/* power_by_squaring (Julia Base intfuncs.jl), used by ω^(-k) in prime.jl:37 */
static cx power_by_squaring(cx x, int64_t p) {
    if (p == 1) return x;
    if (p == 0) return C((REAL)1, (REAL)0);
    if (p == 2) return mul(x, x);
    int t = __builtin_ctzll((unsigned long long)p) + 1;
    p >>= t;
    while ((t -= 1) > 0) x = mul(x, x);
    cx y = x;
    while (p > 0) {
        t = __builtin_ctzll((unsigned long long)p) + 1;
        p >>= t;
        while ((t -= 1) >= 0) x = mul(x, x);
        y = mul(y, x);
    }
    return y;
}
/* inv(z): Julia Base's robust complex inverse (Smith's algorithm; the
 * rescaling branches of Base.inv never trigger for |z| ~ 1). */
static cx cinv(cx z) {
    REAL c = z.re, d = z.im;
    if (fabs((double)c) >= fabs((double)d)) {
        REAL r = d / c;
        REAL t = (REAL)1 / (c + d * r);
        return C(t, -r * t);
    } else {
        REAL cc = d, dd = c;
        REAL r = dd / cc;
        REAL t = (REAL)1 / (cc + dd * r);
        return C(r * t, -t);
    }
}

static node *build_plan(int64_t n) {
    node *nd = (node *)calloc(1, sizeof(node));
    nd->n = n;
    if (n == 1) { nd->kind = K_COPY; return nd; }
    if (is_power_of(n, 2) || is_power_of(n, 3) || is_power_of(n, 5) || is_power_of(n, 7)) {
        /* call_radix_families, NO_FLAG branch (kernel.jl:131-141) */
        static const int r2[3] = {8, 4, 2}, r3[2] = {9, 3}, r5[1] = {5}, r7[1] = {7};
        nd->kind = K_RADIX;
        if (is_power_of(n, 2)) nd->npass = std_radix_plan(n, r2, 3, nd->radix);
        else if (is_power_of(n, 3)) nd->npass = std_radix_plan(n, r3, 2, nd->radix);
        else if (is_power_of(n, 5)) nd->npass = std_radix_plan(n, r5, 1, nd->radix);
        else nd->npass = std_radix_plan(n, r7, 1, nd->radix);
        return nd;
    }
    if (isprime64(n)) {
        /* generate_prime_fft_raders (prime.jl:5-81) */
        nd->kind = K_RADER;
        int64_t g = 0;
        for (int64_t cand = 2; cand < n && !g; cand++) {
            /* smallest generator: cand^i, i=1..n-1, all distinct <=> order n-1 */
            int64_t order_ok = 1, phi = n - 1, f = phi;
            for (int64_t q = 2; q * q <= f; q++) {
                if (f % q == 0) {
                    if (powmod64(cand, phi / q, n) == 1) { order_ok = 0; break; }
                    while (f % q == 0) f /= q;
                }
            }
            if (order_ok && f > 1 && powmod64(cand, phi / f, n) == 1) order_ok = 0;
            if (order_ok) g = cand;
        }
        nd->gen = g;
        int64_t L = n - 1;
        nd->gen_seq = (int64_t *)malloc(sizeof(int64_t) * L);
        nd->inv_seq = (int64_t *)malloc(sizeof(int64_t) * L);
        int64_t inv_gen = powmod64(g, n - 2, n);
        int64_t a = 1, b = 1;
        for (int64_t i = 0; i < L; i++) {
            nd->gen_seq[i] = a; nd->inv_seq[i] = b;
            a = (int64_t)(((__int128)a * g) % n);
            b = (int64_t)(((__int128)b * inv_gen) % n);
        }
        cx omega = cispi_T((REAL)(2.0 / (double)n));      /* ω = cispi(T(2/n)) */
        cx oinv = cinv(omega);
        nd->Wr = (cx *)malloc(sizeof(cx) * L);
        nd->Wr_work = (cx *)malloc(sizeof(cx) * L);
        for (int64_t i = 0; i < L; i++) nd->Wr[i] = power_by_squaring(oinv, nd->inv_seq[i]);
        memcpy(nd->Wr_work, nd->Wr, sizeof(cx) * L);
        nd->F = get_plan(L);
        return nd;
    }
    /* mixed radix (kernel.jl:84-86, mixed_radix.jl:15-28) */
    nd->kind = K_MIXED;
    find_closest_factors(n, &nd->p, &nd->m);
    nd->W = make_D(nd->p, nd->m);
    nd->Fm = get_plan(nd->m);
    nd->Fp = get_plan(nd->p);
    return nd;
}

static node *get_plan(int64_t n) {
    for (node *c = g_cache; c; c = c->next) if (c->n == n) return c;
    node *nd = build_plan(n);
    nd->next = g_cache;
    g_cache = nd;
    return nd;
}

/* Execute: y <- F(x); x may be used as scratch, exactly like the generated
 * closures (radix_exec.jl:105-113) do. */
static void exec(node *nd, cx *y, cx *x);

static void exec_radix(node *nd, cx *y, cx *x) {
    /* Stockham ping-pong as in generate_safe_execute_function! */
    int64_t n = nd->n, s = 1, rem = n;
    cx *in = x, *out = y;
    int eo = 0;
    for (int i = 0; i < nd->npass; i++) {
        int r = nd->radix[i];
        if (i == nd->npass - 1) {
            if (eo) shell_last(r, in, in, s);      /* fft{r}_shell_y!(in, s) */
            else shell_last(r, out, in, s);        /* fft{r}_shell!(out, in, s) */
        } else {
            shell_layered(r, out, in, s, rem / r, 2.0 / (double)rem);
        }
        rem /= r; s *= r; eo = !eo;
        cx *t = in; in = out; out = t;
    }
}

static void exec_mixed(node *nd, cx *y, cx *x) {
    /* generate_formulation_fft closure (mixed_radix.jl:44-78) with per-call
     * scratch in place of the captured Xpm/Ypm (same arithmetic). */
    int64_t p = nd->p, m = nd->m;
    int64_t mx = (p > m) ? p : m;
    cx *Xpm = (cx *)malloc(sizeof(cx) * p * m);    /* column-major p x m */
    cx *Ypm = (cx *)calloc((size_t)(p * m), sizeof(cx));
    cx *ri = (cx *)malloc(sizeof(cx) * mx), *ro = (cx *)malloc(sizeof(cx) * mx);
    memcpy(Xpm, x, sizeof(cx) * p * m);            /* Xpm .= reshape(x, p, m) */
    for (int64_t i = 0; i < p; i++) {              /* Fm over each row i */
        for (int64_t j = 0; j < m; j++) ri[j] = Xpm[i + p * j];
        exec(nd->Fm, ro, ri);
        for (int64_t j = 0; j < m; j++) Ypm[i + p * j] = ro[j];
    }
    for (int64_t i = 1; i <= p - 1; i++)           /* Ypm[i+1, j+1] *= W[j, i] */
        for (int64_t j = 1; j <= m - 1; j++)
            Ypm[i + p * j] = mul(Ypm[i + p * j], nd->W[(i - 1) * (m - 1) + (j - 1)]);
    for (int64_t j = 0; j < m; j++) {              /* Fp over each column j */
        for (int64_t i = 0; i < p; i++) ri[i] = Ypm[i + p * j];
        exec(nd->Fp, ro, ri);
        for (int64_t i = 0; i < p; i++) Xpm[i + p * j] = ro[i];
    }
    for (int64_t l = 0; l < p; l++)                /* y .= vec(transpose(Xpm)) */
        for (int64_t k = 0; k < m; k++) y[k + m * l] = Xpm[l + p * k];
    free(Xpm); free(Ypm); free(ri); free(ro);
}

/* Julia's sum over a Vector: pairwise reduction with a 1024 base block. */
static cx pairwise_sum(const cx *a, int64_t lo, int64_t hi) {
    if (hi - lo < 1024) {
        cx s = a[lo];
        for (int64_t i = lo + 1; i <= hi; i++) s = add(s, a[i]);
        return s;
    }
    int64_t mid = lo + ((hi - lo) >> 1);
    return add(pairwise_sum(a, lo, mid), pairwise_sum(a, mid + 1, hi));
}

static void exec_rader(node *nd, cx *y, cx *x) {
    int64_t n = nd->n, L = n - 1;
    cx *b1 = (cx *)calloc((size_t)L, sizeof(cx)), *b2 = (cx *)calloc((size_t)L, sizeof(cx));
    cx *tmp = (cx *)malloc(sizeof(cx) * L);
    cx x0 = x[0];
    for (int64_t i = 0; i < L; i++) b1[i] = x[nd->gen_seq[i]];      /* prime.jl:54-56 */
    y[0] = add(x0, pairwise_sum(b1, 0, L - 1));                      /* prime.jl:58 */
    exec(nd->F, b2, b1);                                             /* prime.jl:60 */
    if (g_rader_mode == 1) {
        exec(nd->F, b1, nd->Wr_work);      /* faithful: W is F's scratch input */
    } else {
        memcpy(tmp, nd->Wr, sizeof(cx) * L);
        exec(nd->F, b1, tmp);              /* fixed: W copied, never clobbered */
    }
    for (int64_t i = 0; i < L; i++) b2[i] = mul(b2[i], b1[i]);       /* prime.jl:64-66 */
    for (int64_t i = 0; i < L; i++) tmp[i] = conjc(b2[i]);           /* conj.(buffer2) */
    exec(nd->F, b1, tmp);                                            /* prime.jl:69 */
    REAL d = (REAL)(L);
    for (int64_t i = 0; i < L; i++) { cx c = conjc(b1[i]); b1[i] = C(c.re / d, c.im / d); }
    for (int64_t j = 0; j < L; j++) y[nd->inv_seq[j]] = add(x0, b1[j]); /* prime.jl:76-78 */
    free(b1); free(b2); free(tmp);
}

static void exec(node *nd, cx *y, cx *x) {
    switch (nd->kind) {
    case K_COPY: y[0] = x[0]; break;
    case K_RADIX: exec_radix(nd, y, x); break;
    case K_MIXED: exec_mixed(nd, y, x); break;
    case K_RADER: exec_rader(nd, y, x); break;
    }
}

/* ------------------------------ public API -------------------------------- */
/* dir: 0 = fft, 1 = ifft (CatabraFFT.jl:88-101), 2 = bfft (CatabraFFT.jl:103-115) */
static void one_transform(node *nd, int64_t n, const cx *x, cx *y, int dir, cx *ws) {
    memcpy(ws, x, sizeof(cx) * n);                 /* copyto!(workspace.x_work, x) */
    if (dir != 0) for (int64_t i = 0; i < n; i++) ws[i] = conjc(ws[i]);
    exec(nd, y, ws);
    if (dir != 0) for (int64_t i = 0; i < n; i++) y[i] = conjc(y[i]);
    if (dir == 1) {
        REAL d = (REAL)n;
        for (int64_t i = 0; i < n; i++) y[i] = C(y[i].re / d, y[i].im / d);
    }
}

int PFX(set_rader_mode)(int mode) { g_rader_mode = mode; return 0; }

/* Prepare (and cache) the plan tree for n; not thread-safe, call before
 * running batches on several threads. */
int PFX(prepare)(int64_t n) {
    if (n < 1) return -1;
    return get_plan(n) ? 0 : -1;
}

int PFX(fft)(int64_t n, const void *x, void *y, int dir) {
    if (n < 1 || dir < 0 || dir > 2) return -1;
    node *nd = get_plan(n);
    cx *ws = (cx *)malloc(sizeof(cx) * n);
    one_transform(nd, n, (const cx *)x, (cx *)y, dir, ws);
    free(ws);
    return 0;
}

/* Batched driver: transforms [batch][n] contiguous; nthreads <= 0 = all.
 * Each thread uses private scratch (the reference runs one transform per
 * single-threaded process; the arithmetic is identical). */
int PFX(fft_batch)(int64_t n, int64_t batch, const void *x, void *y, int dir, int nthreads) {
    if (n < 1 || batch < 0 || dir < 0 || dir > 2) return -1;
    node *nd = get_plan(n);
    const cx *xc = (const cx *)x;
    cx *yc = (cx *)y;
#ifdef _OPENMP
    int nt = nthreads > 0 ? nthreads : omp_get_max_threads();
    #pragma omp parallel num_threads(nt)
    {
        cx *ws = (cx *)malloc(sizeof(cx) * n);
        #pragma omp for schedule(dynamic, 1)
        for (int64_t b = 0; b < batch; b++) one_transform(nd, n, xc + b * n, yc + b * n, dir, ws);
        free(ws);
    }
#else
    (void)nthreads;
    cx *ws = (cx *)malloc(sizeof(cx) * n);
    for (int64_t b = 0; b < batch; b++) one_transform(nd, n, xc + b * n, yc + b * n, dir, ws);
    free(ws);
#endif
    return 0;
}

int PFX(max_threads)(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* Human-readable plan tree, e.g. "mixed(32,945)[radix(8,4);mixed(27,35)[...]]". */
static int describe(node *nd, char *buf, int len) {
    int w = 0;
#define APP(...) do { int k = snprintf(buf + w, (w < len) ? (size_t)(len - w) : 0, __VA_ARGS__); w += k; } while (0)
    switch (nd->kind) {
    case K_COPY: APP("copy"); break;
    case K_RADIX:
        APP("radix(");
        for (int i = 0; i < nd->npass; i++) APP(i ? ",%d" : "%d", nd->radix[i]);
        APP(")");
        break;
    case K_MIXED:
        APP("mixed(%lld,%lld)[", (long long)nd->p, (long long)nd->m);
        w += describe(nd->Fm, buf + w, (w < len) ? len - w : 0);
        APP(";");
        w += describe(nd->Fp, buf + w, (w < len) ? len - w : 0);
        APP("]");
        break;
    case K_RADER:
        APP("rader(%lld,g=%lld)[", (long long)nd->n, (long long)nd->gen);
        w += describe(nd->F, buf + w, (w < len) ? len - w : 0);
        APP("]");
        break;
    }
#undef APP
    return w;
}
int PFX(describe)(int64_t n, char *buf, int len) {
    if (n < 1 || len < 1) return -1;
    node *nd = get_plan(n);
    buf[0] = 0;
    describe(nd, buf, len);
    return 0;
}

/* Explicit Stockham plan execution (used to check individual codelets). */
int PFX(radix_plan_exec)(int64_t n, const int *radices, int np, const void *x, void *y) {
    node nd;
    memset(&nd, 0, sizeof nd);
    nd.kind = K_RADIX; nd.n = n; nd.npass = np;
    int64_t prod = 1;
    for (int i = 0; i < np; i++) { nd.radix[i] = radices[i]; prod *= radices[i]; }
    if (prod != n || np > MAXPASS) return -1;
    cx *ws = (cx *)malloc(sizeof(cx) * n);
    memcpy(ws, x, sizeof(cx) * n);
    exec_radix(&nd, (cx *)y, ws);
    free(ws);
    return 0;
}

int PFX(find_closest_factors)(int64_t n, int64_t *p, int64_t *m) {
    find_closest_factors(n, p, m);
    return 0;
}

int64_t PFX(rader_generator)(int64_t n) {
    if (!isprime64(n) || n < 3) return -1;
    node *nd = get_plan(n);
    return nd->kind == K_RADER ? nd->gen : -1;
}

void PFX(empty_cache)(void) {
    /* leak-free teardown is not needed for a test oracle; drop the chain */
    g_cache = NULL;
}
