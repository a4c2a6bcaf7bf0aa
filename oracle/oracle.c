/*
 * oracle.c -- FP64 CPU restatement of IQ-TREE's reversible Felsenstein likelihood path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA kernels in gems_b200, and the
 * "port" CPU baseline that bench.py times.  The product never links or calls this file.
 *
 * What is restated (paths relative to the IQ-TREE 3 source tree):
 *   tree/phylokernelnew.h:900-1114   computePartialInfo (E(t) = evec*exp(eval*r*t), tip tables)
 *   tree/phylokernelnew.h:1293-2043  computePartialLikelihoodSIMD: tip-tip, tip-internal,
 *                                    internal-internal, NORM and SAFE 2^-256 scaling
 *   tree/phylokernelnew.h:2053-2235  computeLikelihoodBufferSIMD (theta, buffer_scale_all)
 *   tree/phylokernelnew.h:2238-2650  computeLikelihoodDervSIMD (lh, df, ddf, G_matrix row)
 *   tree/phylokernelnew.h:2658-3275  computeLikelihoodBranchSIMD (pattern lnL, SAFE min-scale,
 *                                    non-finite fix-up)
 *   tree/phylokernelnew.h:3285-3495  computeLikelihoodFromBufferSIMD
 *   tree/phylotreesse.cpp:243-612    tip partial likelihoods, ptn_freq, ptn_invar
 *   tree/phylotree.cpp:1258,2540-2800,6031  computeLikelihood, computeFuncDerv,
 *                                    optimizeOneBranch, optimizeAllBranches, traversal
 *   tree/mtree.cpp:3040-3082         findFarthestLeaf, getPreOrderBranches
 *   utils/optimization.cpp:422-499   minimizeNewton
 *   utils/eigendecomposition.cpp     eigensystem_sym (tred2 + tqli, published Householder / QL)
 *   model/rategamma.cpp:98-478       discrete Gamma rates (published AS91 / AS32 / AS70 /
 *                                    Pike-Hill log-gamma algorithms, restated)
 * Only reversible models, binary trees and the non-site-specific, non-mixture kernel are
 * covered; +ASC and robust-phylo modes are not part of the path.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_SCALE_EXP 256
#define ORC_SCALE_THR 8.636168555094444625386e-78 /* 2^-256 */
#define ORC_LOG_SCALE_THR (-177.4456782233459932741)
#define ORC_ZERO_FREQ 1e-10

static int g_threads = 1;
void orc_set_threads(int nthreads) { g_threads = nthreads > 0 ? nthreads : 1; }

/* ===================================================================== */
/* Discrete Gamma rates                                                  */
/* ===================================================================== */

/* ln Gamma(a), Pike & Hill (1966) ACM Alg. 291 with Stirling's series. */
static double lngamma_ph(double a) {
    double x = a, f = 0.0, z;
    if (x < 7) {
        f = 1;
        z = x - 1;
        while (++z < 7) f *= z;
        x = z;
        f = -log(f);
    }
    z = 1 / (x * x);
    return f + (x - 0.5) * log(x) - x + .918938533204673 +
           (((-.000595238095238 * z + .000793650793651) * z - .002777777777778) * z +
            .083333333333333) / x;
}

/* Incomplete gamma ratio I(x, p), Bhattacharjee (1970) AS32: series for x<=1 or x<p,
 * continued fraction otherwise. */
static double incgamma_as32(double x, double p, double lng) {
    const double acc = 1e-8, big = 1e30;
    double factor, gin, rn, term, a, b, an, dif, pn[6];
    int i;
    if (x == 0) return 0;
    if (x < 0 || p <= 0) return -1;
    factor = exp(p * log(x) - x - lng);
    if (!(x > 1 && x >= p)) {
        gin = 1;
        term = 1;
        rn = p;
        do {
            rn += 1;
            term *= x / rn;
            gin += term;
        } while (term > acc);
        return gin * factor / p;
    }
    a = 1 - p;
    b = a + x + 1;
    term = 0;
    pn[0] = 1;
    pn[1] = x;
    pn[2] = x + 1;
    pn[3] = x * b;
    gin = pn[2] / pn[3];
    for (;;) {
        a += 1;
        b += 2;
        term += 1;
        an = a * term;
        for (i = 0; i < 2; i++) pn[i + 4] = b * pn[i + 2] - an * pn[i];
        if (pn[5] != 0) {
            rn = pn[4] / pn[5];
            dif = fabs(gin - rn);
            if (dif <= acc && dif <= acc * rn) return 1 - factor * gin;
            gin = rn;
        }
        for (i = 0; i < 4; i++) pn[i] = pn[i + 2];
        if (fabs(pn[4]) >= big)
            for (i = 0; i < 4; i++) pn[i] /= big;
    }
}

/* Normal percentage point, Odeh & Evans (1974) AS70. */
static double pointnormal_as70(double prob) {
    const double a0 = -.322232431088, a1 = -1, a2 = -.342242088547, a3 = -.0204231210245;
    const double a4 = -.453642210148e-4, b0 = .0993484626060, b1 = .588581570495;
    const double b2 = .531103462366, b3 = .103537752850, b4 = .0038560700634;
    double p1 = prob < 0.5 ? prob : 1 - prob, y, z;
    if (p1 < 1e-20) return -9999;
    y = sqrt(log(1 / (p1 * p1)));
    z = y + ((((y * a4 + a3) * y + a2) * y + a1) * y + a0) /
                ((((y * b4 + b3) * y + b2) * y + b1) * y + b0);
    return prob < 0.5 ? -z : z;
}

/* Chi-square percentage point, Best & Roberts (1975) AS91. */
static double pointchi2_as91(double p, double v) {
    const double e = .5e-6, aa = .6931471805;
    double g, xx, c, ch, a, q, p1, p2, t, x, b, s1, s2, s3, s4, s5, s6;
    if (p < .000002 || p > .999998 || v <= 0) return -1;
    g = lngamma_ph(v / 2);
    xx = v / 2;
    c = xx - 1;
    if (v < -1.24 * log(p)) {
        ch = pow(p * xx * exp(g + xx * aa), 1 / xx);
        if (ch - e < 0) return ch;
    } else if (v <= .32) {
        ch = 0.4;
        a = log(1 - p);
        do {
            q = ch;
            p1 = 1 + ch * (4.67 + ch);
            p2 = ch * (6.73 + ch * (6.66 + ch));
            t = -0.5 + (4.67 + 2 * ch) / p1 - (6.73 + ch * (13.32 + 3 * ch)) / p2;
            ch -= (1 - exp(a + g + .5 * ch + c * aa) * p2 / p1) / t;
        } while (fabs(q / ch - 1) - .01 > 0);
    } else {
        x = pointnormal_as70(p);
        p1 = 0.222222 / v;
        ch = v * pow(x * sqrt(p1) + 1 - p1, 3.0);
        if (ch > 2.2 * v + 6) ch = -2 * (log(1 - p) - c * log(.5 * ch) + g);
    }
    do {
        q = ch;
        p1 = .5 * ch;
        t = incgamma_as32(p1, xx, g);
        if (t < 0) return -1;
        p2 = p - t;
        t = p2 * exp(xx * aa + g + p1 - c * log(ch));
        b = t / ch;
        a = 0.5 * t - b * c;
        s1 = (210 + a * (140 + a * (105 + a * (84 + a * (70 + 60 * a))))) / 420;
        s2 = (420 + a * (735 + a * (966 + a * (1141 + 1278 * a)))) / 2520;
        s3 = (210 + a * (462 + a * (707 + 932 * a))) / 2520;
        s4 = (252 + a * (672 + 1182 * a) + c * (294 + a * (889 + 1740 * a))) / 5040;
        s5 = (84 + 264 * a + c * (175 + 606 * a)) / 2520;
        s6 = (120 + c * (346 + 127 * c)) / 5040;
        ch += t * (1 + 0.5 * t * s1 - b * c * (s1 - b * (s2 - b * (s3 - b * (s4 - b * (s5 - b * s6))))));
    } while (fabs(q / ch - 1) > e);
    return ch;
}

void orc_gamma_rates(double alpha, int ncat, int cut_median, double *rates) {
    int i;
    if (ncat == 1) {
        rates[0] = 1.0;
        return;
    }
    /* RateGamma starts with rates[]=1/ncat... the rescale below uses the sum before and after;
     * the constructor's initial rates sum to ncat (all 1.0), rategamma.cpp:98-150. */
    double cur_scale = (double)ncat;
    if (!cut_median) {
        double lnga1 = lngamma_ph(alpha + 1);
        double *fk = (double *)malloc(sizeof(double) * ncat);
        for (i = 0; i < ncat - 1; i++)
            fk[i] = pointchi2_as91((i + 1.0) / ncat, 2.0 * alpha) / (2.0 * alpha);
        for (i = 0; i < ncat - 1; i++) fk[i] = incgamma_as32(fk[i] * alpha, alpha + 1, lnga1);
        rates[0] = fk[0] * ncat;
        rates[ncat - 1] = (1 - fk[ncat - 2]) * ncat;
        for (i = 1; i < ncat - 1; i++) rates[i] = (fk[i] - fk[i - 1]) * ncat;
        free(fk);
    } else {
        double sum = 0;
        for (i = 0; i < ncat; i++) {
            double prob = (2.0 * i + 1) / (2.0 * ncat);
            double pp = pointchi2_as91(prob, 2.0 * alpha) / (2.0 * alpha);
            rates[i] = pp < 0 ? -pp : pp;
        }
        for (i = 0; i < ncat; i++) sum += rates[i];
        for (i = 0; i < ncat; i++) rates[i] = rates[i] * ncat / sum;
    }
    double new_scale = 0;
    for (i = 0; i < ncat; i++) new_scale += rates[i];
    if (new_scale != cur_scale)
        for (i = 0; i < ncat; i++) rates[i] *= cur_scale / new_scale;
}

/* ===================================================================== */
/* Eigensystem: normalised Q -> drop zero-frequency states -> symmetrise  */
/* with sqrt(pi) -> Householder tridiagonalisation -> implicit QL.        */
/* ===================================================================== */

static void house_tridiag(double **a, int n, double *d, double *e) {
    int l, k, j, i;
    double scale, hh, h, g, f;
    for (i = n - 1; i > 0; i--) {
        l = i - 1;
        h = scale = 0.0;
        if (l > 0) {
            for (k = 0; k <= l; k++) scale += fabs(a[i][k]);
            if (scale == 0.0) {
                e[i] = a[i][l];
            } else {
                for (k = 0; k <= l; k++) {
                    a[i][k] /= scale;
                    h += a[i][k] * a[i][k];
                }
                f = a[i][l];
                g = (f >= 0.0 ? -sqrt(h) : sqrt(h));
                e[i] = scale * g;
                h -= f * g;
                a[i][l] = f - g;
                f = 0.0;
                for (j = 0; j <= l; j++) {
                    a[j][i] = a[i][j] / h;
                    g = 0.0;
                    for (k = 0; k <= j; k++) g += a[j][k] * a[i][k];
                    for (k = j + 1; k <= l; k++) g += a[k][j] * a[i][k];
                    e[j] = g / h;
                    f += e[j] * a[i][j];
                }
                hh = f / (h + h);
                for (j = 0; j <= l; j++) {
                    f = a[i][j];
                    e[j] = g = e[j] - hh * f;
                    for (k = 0; k <= j; k++) a[j][k] -= (f * e[k] + g * a[i][k]);
                }
            }
        } else {
            e[i] = a[i][l];
        }
        d[i] = h;
    }
    d[0] = 0.0;
    e[0] = 0.0;
    for (i = 0; i < n; i++) {
        l = i;
        if (d[i] != 0.0) {
            for (j = 0; j < l; j++) {
                g = 0.0;
                for (k = 0; k < l; k++) g += a[i][k] * a[k][j];
                for (k = 0; k < l; k++) a[k][j] -= g * a[k][i];
            }
        }
        d[i] = a[i][i];
        a[i][i] = 1.0;
        for (j = 0; j < l; j++) a[j][i] = a[i][j] = 0.0;
    }
}

static double hypot_safe(double a, double b) {
    double x = fabs(a), y = fabs(b);
    if (x > y) {
        double r = y / x;
        return x * sqrt(1.0 + (r == 0.0 ? 0.0 : r * r));
    }
    if (y == 0.0) return 0.0;
    double r = x / y;
    return y * sqrt(1.0 + (r == 0.0 ? 0.0 : r * r));
}

static void ql_implicit(double *d, double *e, int n, double **z) {
    int m, l, iter, i, k;
    double s, r, p, g, f, dd, c, b;
    for (i = 1; i < n; i++) e[i - 1] = e[i];
    e[n - 1] = 0.0;
    for (l = 0; l < n; l++) {
        iter = 0;
        do {
            for (m = l; m < n - 1; m++) {
                dd = fabs(d[m]) + fabs(d[m + 1]);
                if ((double)(fabs(e[m]) + dd) == dd) break;
            }
            if (m != l) {
                if (iter++ == 100) break;
                g = (d[l + 1] - d[l]) / (2.0 * e[l]);
                r = hypot_safe(g, 1.0);
                g = d[m] - d[l] + e[l] / (g + (g >= 0.0 ? fabs(r) : -fabs(r)));
                s = c = 1.0;
                p = 0.0;
                for (i = m - 1; i >= l; i--) {
                    f = s * e[i];
                    b = c * e[i];
                    e[i + 1] = (r = hypot_safe(f, g));
                    if (r == 0.0) {
                        d[i + 1] -= p;
                        e[m] = 0.0;
                        break;
                    }
                    s = f / r;
                    c = g / r;
                    g = d[i + 1] - p;
                    r = (d[i] - g) * s + 2.0 * c * b;
                    d[i + 1] = g + (p = s * r);
                    g = c * r - b;
                    for (k = 0; k < n; k++) {
                        f = z[k][i + 1];
                        z[k][i + 1] = s * z[k][i] + c * f;
                        z[k][i] = c * z[k][i] - s * f;
                    }
                }
                if (r == 0.0 && i >= l) continue;
                d[l] -= p;
                e[l] = g;
                e[m] = 0.0;
            }
        } while (m != l);
    }
}

int orc_eigensystem_sym(int n, const double *rates_upper, const double *freq, double *eval,
                        double *evec, double *inv_evec) {
    int i, j, k, nn = 0;
    double *forg = (double *)calloc(n, sizeof(double));
    double *nforg = (double *)calloc(n, sizeof(double));
    double *fsq = (double *)calloc(n, sizeof(double));
    double *offd = (double *)calloc(n, sizeof(double));
    double *ev = (double *)calloc(n, sizeof(double));
    double *m = (double *)calloc(n, sizeof(double));
    double **a = (double **)malloc(sizeof(double *) * n);
    double **b = (double **)malloc(sizeof(double *) * n);
    for (i = 0; i < n; i++) {
        a[i] = (double *)calloc(n, sizeof(double));
        b[i] = (double *)calloc(n, sizeof(double));
    }
    double sum = 0;
    for (i = 0; i < n; i++) sum += freq[i];
    sum = 1.0 / sum;
    for (i = 0; i < n; i++) forg[i] = freq[i] * sum;
    /* half matrix -> symmetric exchangeabilities, zero for zero-frequency states
     * (modelmarkov.cpp:1605-1632) */
    for (i = 0, k = 0; i < n; i++) {
        a[i][i] = 0.0;
        for (j = i + 1; j < n; j++, k++) {
            double r = (freq[i] <= ORC_ZERO_FREQ || freq[j] <= ORC_ZERO_FREQ) ? 0 : rates_upper[k];
            a[i][j] = a[j][i] = r;
        }
    }
    /* computeRateMatrix: q_ij = pi_j * s_ij, rows sum to zero, mean rate normalised to 1 */
    for (i = 0; i < n; i++)
        for (j = 0; j < n; j++) a[i][j] = forg[j] * a[i][j];
    double tot = 0;
    for (i = 0; i < n; i++) {
        double t = 0;
        for (j = 0; j < n; j++)
            if (j != i) t += a[i][j];
        m[i] = t;
        tot += t * forg[i];
    }
    double delta = 1.0 / tot;
    for (i = 0; i < n; i++)
        for (j = 0; j < n; j++) a[i][j] = (i != j) ? delta * a[i][j] : delta * (-m[i]);
    for (i = 0; i < n; i++)
        for (j = 0; j < n; j++) b[i][j] = a[i][j];
    /* eliminateZero */
    for (i = 0; i < n; i++)
        if (forg[i] > ORC_ZERO_FREQ) nforg[nn++] = forg[i];
    if (nn != n) {
        int inew = 0;
        for (i = 0; i < n; i++) {
            if (forg[i] > ORC_ZERO_FREQ) {
                int jnew = 0;
                for (j = 0; j < n; j++)
                    if (forg[j] > ORC_ZERO_FREQ) a[inew][jnew++] = b[i][j];
                inew++;
            }
        }
    }
    /* symmetrise: a_ji *= sqrt(pi_j)/sqrt(pi_i) for j<i, mirrored */
    for (i = 0; i < nn; i++) fsq[i] = sqrt(nforg[i]);
    for (i = 0; i < nn; i++) {
        double tmp = 1.0 / fsq[i];
        for (j = 0; j < i; j++) {
            a[j][i] *= fsq[j] * tmp;
            a[i][j] = a[j][i];
        }
    }
    house_tridiag(a, nn, ev, offd);
    ql_implicit(ev, offd, nn, a);
    int inew = nn - 1;
    for (i = n - 1; i >= 0; i--) eval[i] = (forg[i] > ORC_ZERO_FREQ) ? ev[inew--] : 0;
    inew = nn - 1;
    for (i = n - 1; i >= 0; i--) {
        if (forg[i] > ORC_ZERO_FREQ) {
            int jnew = nn - 1;
            for (j = n - 1; j >= 0; j--) {
                if (forg[j] > ORC_ZERO_FREQ) {
                    evec[i * n + j] = a[inew][jnew] / fsq[inew];
                    inv_evec[i * n + j] = a[jnew][inew] * fsq[jnew];
                    jnew--;
                } else {
                    evec[i * n + j] = (i == j);
                    inv_evec[i * n + j] = (i == j);
                }
            }
            inew--;
        } else {
            for (j = 0; j < n; j++) evec[i * n + j] = inv_evec[i * n + j] = (i == j);
        }
    }
    int bad = 0;
    for (i = 0; i < nn; i++)
        if (ev[i] > 0.01) bad = 1;
    for (i = 0; i < n; i++) {
        free(a[i]);
        free(b[i]);
    }
    free(a);
    free(b);
    free(forg);
    free(nforg);
    free(fsq);
    free(offd);
    free(ev);
    free(m);
    return bad;
}

/* ===================================================================== */
/* Tree session                                                          */
/* ===================================================================== */

struct orc_tree {
    int ntaxa, nnode, nedges;
    int n, ncat, block, safe, unknown;
    int *deg, *adj;      /* adj[u*3+k]: k-th neighbour of u */
    double *len;         /* len[u*3+k] (mirrors both directions) */
    int *eu, *ev;
    /* directed branch d = u*3+k: u -> adj[u*3+k], holds the subtree hanging at adj[u*3+k] */
    double **plh;
    uint16_t **scl;
    unsigned char *computed;
    /* model */
    double *eval, *evec, *inv_evec, *rates, *props, *freq_state, p_invar;
    double *tip; /* [(unknown+1)][n] eigen-space tip vectors */
    /* patterns */
    int nptn, nptn_pad;
    uint8_t *states; /* [ntaxa][nptn_pad] */
    double *ptn_freq, *ptn_invar;
    /* buffers */
    double *theta, *scale_all, *G, *plh_out;
    int theta_computed;
    int cur_u, cur_k; /* current_it = directed u -> adj[u*3+k] */
    double min_bl, max_bl;
    long long partial_ops;
    int newton_evals;
};

static int find_nei(const orc_tree *t, int u, int v) {
    for (int k = 0; k < t->deg[u]; k++)
        if (t->adj[u * 3 + k] == v) return k;
    return -1;
}
static int is_leaf(const orc_tree *t, int u) { return t->deg[u] == 1; }

orc_tree *orc_tree_new(int ntaxa, int nedges, const int *eu, const int *ev, const double *elen,
                       int nstates, int ncat, int safe) {
    orc_tree *t = (orc_tree *)calloc(1, sizeof(orc_tree));
    int nnode = nedges + 1, i;
    t->ntaxa = ntaxa;
    t->nnode = nnode;
    t->nedges = nedges;
    t->n = nstates;
    t->ncat = ncat;
    t->block = nstates * ncat;
    t->safe = safe;
    t->unknown = (nstates == 4) ? 18 : (nstates == 20) ? 23 : nstates;
    t->deg = (int *)calloc(nnode, sizeof(int));
    t->adj = (int *)malloc(sizeof(int) * nnode * 3);
    t->len = (double *)calloc(nnode * 3, sizeof(double));
    t->eu = (int *)malloc(sizeof(int) * nedges);
    t->ev = (int *)malloc(sizeof(int) * nedges);
    for (i = 0; i < nnode * 3; i++) t->adj[i] = -1;
    for (i = 0; i < nedges; i++) {
        int u = eu[i], v = ev[i];
        t->eu[i] = u;
        t->ev[i] = v;
        if (t->deg[u] >= 3 || t->deg[v] >= 3) {
            orc_tree_free(t);
            return NULL;
        }
        t->adj[u * 3 + t->deg[u]] = v;
        t->len[u * 3 + t->deg[u]] = elen[i];
        t->deg[u]++;
        t->adj[v * 3 + t->deg[v]] = u;
        t->len[v * 3 + t->deg[v]] = elen[i];
        t->deg[v]++;
    }
    t->plh = (double **)calloc(nnode * 3, sizeof(double *));
    t->scl = (uint16_t **)calloc(nnode * 3, sizeof(uint16_t *));
    t->computed = (unsigned char *)calloc(nnode * 3, 1);
    t->cur_u = -1;
    t->min_bl = 1e-6;
    t->max_bl = 10.0;
    return t;
}

void orc_tree_free(orc_tree *t) {
    if (!t) return;
    if (t->plh)
        for (int i = 0; i < t->nnode * 3; i++) {
            free(t->plh[i]);
            free(t->scl[i]);
        }
    free(t->plh);
    free(t->scl);
    free(t->computed);
    free(t->deg);
    free(t->adj);
    free(t->len);
    free(t->eu);
    free(t->ev);
    free(t->eval);
    free(t->evec);
    free(t->inv_evec);
    free(t->rates);
    free(t->props);
    free(t->freq_state);
    free(t->tip);
    free(t->states);
    free(t->ptn_freq);
    free(t->ptn_invar);
    free(t->theta);
    free(t->scale_all);
    free(t->G);
    free(t->plh_out);
    free(t);
}

void orc_clear_all_partial_lh(orc_tree *t) {
    memset(t->computed, 0, t->nnode * 3);
    t->theta_computed = 0;
}

static double *dup(const double *p, int n) {
    double *q = (double *)malloc(sizeof(double) * n);
    memcpy(q, p, sizeof(double) * n);
    return q;
}

/* tip table: tip[state][i] = sum_j inv_evec[i][j] * ind(state, j)
 * (phylotreesse.cpp:361-371 with modelsubst.cpp:183-208, modeldna.cpp:462-474,
 *  modelprotein.cpp:1240-1255) */
static void build_tip(orc_tree *t) {
    int n = t->n, s, i, j;
    free(t->tip);
    t->tip = (double *)calloc((size_t)(t->unknown + 1) * n, sizeof(double));
    double *ind = (double *)malloc(sizeof(double) * n);
    for (s = 0; s <= t->unknown; s++) {
        for (j = 0; j < n; j++) ind[j] = 0;
        if (s < n) {
            ind[s] = 1;
        } else if (n == 4 && s < 18) {
            int cs = s - n + 1;
            for (j = 0; j < 4; j++)
                if (cs & (1 << j)) ind[j] = 1;
        } else if (n == 20 && s < 23) {
            static const int amb[3][2] = {{2, 3}, {5, 6}, {9, 10}};
            ind[amb[s - 20][0]] = 1;
            ind[amb[s - 20][1]] = 1;
        } else {
            for (j = 0; j < n; j++) ind[j] = 1;
        }
        for (i = 0; i < n; i++) {
            double acc = 0;
            for (j = 0; j < n; j++) acc += t->inv_evec[i * n + j] * ind[j];
            t->tip[s * n + i] = acc;
        }
    }
    free(ind);
}

static void compute_ptn_invar(orc_tree *t, const uint8_t *const_char) {
    int p, x;
    for (p = 0; p < t->nptn_pad; p++) t->ptn_invar[p] = 0.0;
    if (t->p_invar == 0.0 || !t->freq_state) return;
    for (p = 0; p < t->nptn; p++) {
        int cc = const_char ? const_char[p] : t->unknown + 1;
        if (cc > t->unknown) continue;
        if (cc == t->unknown) {
            t->ptn_invar[p] = t->p_invar;
        } else if (cc < t->n) {
            t->ptn_invar[p] = t->p_invar * t->freq_state[cc];
        } else if (t->n == 4) {
            int cs = cc - t->n + 1;
            double acc = 0;
            for (x = 0; x < 4; x++)
                if (cs & (1 << x)) acc += t->freq_state[x];
            t->ptn_invar[p] = acc * t->p_invar;
        } else if (t->n == 20) {
            static const int amb[3] = {4 + 8, 32 + 64, 512 + 1024};
            double acc = 0;
            for (x = 0; x < 11; x++)
                if (amb[cc - 20] & (1 << x)) acc += t->freq_state[x];
            t->ptn_invar[p] = acc * t->p_invar;
        }
    }
    for (p = t->nptn; p < t->nptn_pad; p++) t->ptn_invar[p] = t->p_invar;
}

void orc_set_model(orc_tree *t, const double *eval, const double *evec, const double *inv_evec,
                   const double *rates, const double *props, double p_invar,
                   const double *state_freq) {
    int n = t->n;
    free(t->eval);
    free(t->evec);
    free(t->inv_evec);
    free(t->rates);
    free(t->props);
    free(t->freq_state);
    t->eval = dup(eval, n);
    t->evec = dup(evec, n * n);
    t->inv_evec = dup(inv_evec, n * n);
    t->rates = dup(rates, t->ncat);
    t->props = dup(props, t->ncat);
    t->freq_state = state_freq ? dup(state_freq, n) : NULL;
    t->p_invar = p_invar;
    build_tip(t);
    orc_clear_all_partial_lh(t);
}

void orc_set_patterns(orc_tree *t, int nptn, const uint8_t *states, const double *freq,
                      const uint8_t *const_char) {
    int i, p;
    t->nptn = nptn;
    t->nptn_pad = (nptn + 3) & ~3;
    free(t->states);
    free(t->ptn_freq);
    free(t->ptn_invar);
    free(t->theta);
    free(t->scale_all);
    free(t->G);
    free(t->plh_out);
    t->states = (uint8_t *)malloc((size_t)t->ntaxa * t->nptn_pad);
    for (i = 0; i < t->ntaxa; i++) {
        memcpy(t->states + (size_t)i * t->nptn_pad, states + (size_t)i * nptn, nptn);
        for (p = nptn; p < t->nptn_pad; p++) t->states[(size_t)i * t->nptn_pad + p] = t->unknown;
    }
    t->ptn_freq = (double *)calloc(t->nptn_pad, sizeof(double));
    for (p = 0; p < nptn; p++) t->ptn_freq[p] = freq[p];
    t->ptn_invar = (double *)calloc(t->nptn_pad, sizeof(double));
    compute_ptn_invar(t, const_char);
    t->theta = (double *)calloc((size_t)t->nptn_pad * t->block, sizeof(double));
    t->scale_all = (double *)calloc(t->nptn_pad, sizeof(double));
    t->G = (double *)calloc(t->nptn_pad, sizeof(double));
    t->plh_out = (double *)calloc(t->nptn_pad, sizeof(double));
    for (i = 0; i < t->nnode * 3; i++) {
        free(t->plh[i]);
        free(t->scl[i]);
        t->plh[i] = NULL;
        t->scl[i] = NULL;
    }
    orc_clear_all_partial_lh(t);
}

void orc_set_branch_limits(orc_tree *t, double min_bl, double max_bl) {
    t->min_bl = min_bl;
    t->max_bl = max_bl;
}

int orc_set_length(orc_tree *t, int u, int v, double len) {
    int ku = find_nei(t, u, v), kv = find_nei(t, v, u);
    if (ku < 0 || kv < 0) return -1;
    t->len[u * 3 + ku] = len;
    t->len[v * 3 + kv] = len;
    return 0;
}
double orc_get_length(orc_tree *t, int u, int v) {
    int k = find_nei(t, u, v);
    return k < 0 ? -1.0 : t->len[u * 3 + k];
}
void orc_get_lengths(orc_tree *t, double *out) {
    for (int i = 0; i < t->nedges; i++) out[i] = orc_get_length(t, t->eu[i], t->ev[i]);
}

/* clearReversePartialLh (tree/phylonode.cpp:22): invalidate every directed branch that
 * points back towards `dad` from the subtree at `node`. */
static void clear_reverse(orc_tree *t, int node, int dad) {
    for (int k = 0; k < t->deg[node]; k++) {
        int c = t->adj[node * 3 + k];
        if (c == dad) continue;
        int kb = find_nei(t, c, node);
        t->computed[c * 3 + kb] = 0;
        clear_reverse(t, c, node);
    }
}

/* ---- partial likelihood of one directed branch (dad -> node) ---------------------- */

/* echild[c][x][i] = evec[x][i] * exp(eval[i] * rate_c * len)   (phylokernelnew.h:1043-1062) */
static void make_echild(const orc_tree *t, double len, double *e) {
    int n = t->n, c, x, i;
    double *ex = (double *)malloc(sizeof(double) * n);
    for (c = 0; c < t->ncat; c++) {
        double lc = t->rates[c] * len;
        for (i = 0; i < n; i++) ex[i] = exp(t->eval[i] * lc);
        for (x = 0; x < n; x++)
            for (i = 0; i < n; i++) e[(c * n + x) * n + i] = t->evec[x * n + i] * ex[i];
    }
    free(ex);
}

/* leaf[state][c][x] = sum_i echild[c][x][i] * tip[state][i], unknown row = 1.0
 * (phylokernelnew.h:1064-1088) */
static void make_leaf(const orc_tree *t, const double *e, double *leaf) {
    int n = t->n, s, c, x, i, blk = t->block;
    for (s = 0; s < t->unknown; s++)
        for (c = 0; c < t->ncat; c++)
            for (x = 0; x < n; x++) {
                double acc = 0;
                for (i = 0; i < n; i++) acc += e[(c * n + x) * n + i] * t->tip[s * n + i];
                leaf[s * blk + c * n + x] = acc;
            }
    for (x = 0; x < blk; x++) leaf[t->unknown * blk + x] = 1.0;
}

static void ensure_buffer(orc_tree *t, int d) {
    if (!t->plh[d]) {
        t->plh[d] = (double *)calloc((size_t)t->nptn_pad * t->block, sizeof(double));
        t->scl[d] = (uint16_t *)calloc((size_t)t->nptn_pad * (t->safe ? t->ncat : 1), 2);
    }
}

static void compute_partial(orc_tree *t, int dad, int node) {
    const int n = t->n, ncat = t->ncat, blk = t->block, safe = t->safe;
    int d = dad * 3 + find_nei(t, dad, node);
    int left = -1, right = -1, kk;
    for (kk = 0; kk < t->deg[node]; kk++) {
        int c = t->adj[node * 3 + kk];
        if (c == dad) continue;
        if (left < 0) left = c;
        else right = c;
    }
    /* tip-internal: make the tip the left child (phylokernelnew.h:1394-1406) */
    if (!is_leaf(t, left) && is_leaf(t, right)) {
        int tmp = left;
        left = right;
        right = tmp;
    }
    int dl = node * 3 + find_nei(t, node, left), dr = node * 3 + find_nei(t, node, right);
    double *eL = (double *)malloc(sizeof(double) * ncat * n * n);
    double *eR = (double *)malloc(sizeof(double) * ncat * n * n);
    make_echild(t, t->len[dl], eL);
    make_echild(t, t->len[dr], eR);
    double *leafL = NULL, *leafR = NULL;
    if (is_leaf(t, left)) {
        leafL = (double *)malloc(sizeof(double) * (t->unknown + 1) * blk);
        make_leaf(t, eL, leafL);
    }
    if (is_leaf(t, right)) {
        leafR = (double *)malloc(sizeof(double) * (t->unknown + 1) * blk);
        make_leaf(t, eR, leafR);
    }
    ensure_buffer(t, d);
    double *out = t->plh[d];
    uint16_t *sdad = t->scl[d];
    const double *L = is_leaf(t, left) ? NULL : t->plh[dl];
    const double *R = is_leaf(t, right) ? NULL : t->plh[dr];
    const uint16_t *sL = L ? t->scl[dl] : NULL, *sR = R ? t->scl[dr] : NULL;
    const uint8_t *stL = leafL ? t->states + (size_t)left * t->nptn_pad : NULL;
    const uint8_t *stR = leafR ? t->states + (size_t)right * t->nptn_pad : NULL;
    const int P = t->nptn_pad;
    const int nsc = safe ? ncat : 1;

#pragma omp parallel for schedule(static) num_threads(g_threads)
    for (int p = 0; p < P; p++) {
        double tmp[64];
        double *o = out + (size_t)p * blk;
        const double *lp = L ? L + (size_t)p * blk : leafL + (size_t)stL[p] * blk;
        const double *rp = R ? R + (size_t)p * blk : leafR + (size_t)stR[p] * blk;
        uint16_t *sd = sdad + (size_t)p * nsc;
        double lh_max = 0.0;
        int c, x, i, j;
        if (!safe) sd[0] = (uint16_t)((sL ? sL[p] : 0) + (sR ? sR[p] : 0));
        for (c = 0; c < ncat; c++) {
            if (safe) {
                lh_max = 0.0;
                sd[c] = (uint16_t)((sL ? sL[(size_t)p * ncat + c] : 0) +
                                   (sR ? sR[(size_t)p * ncat + c] : 0));
            }
            for (x = 0; x < n; x++) {
                double vl, vr;
                if (L) {
                    vl = 0;
                    for (i = 0; i < n; i++) vl += eL[(c * n + x) * n + i] * lp[c * n + i];
                } else {
                    vl = lp[c * n + x];
                }
                if (R) {
                    vr = 0;
                    for (i = 0; i < n; i++) vr += eR[(c * n + x) * n + i] * rp[c * n + i];
                } else {
                    vr = rp[c * n + x];
                }
                tmp[x] = vl * vr;
            }
            for (j = 0; j < n; j++) {
                double acc = 0;
                for (x = 0; x < n; x++) acc += t->inv_evec[j * n + x] * tmp[x];
                o[c * n + j] = acc;
                double a = fabs(acc);
                if (a > lh_max) lh_max = a;
            }
            /* tip-tip partials are never scaled (phylokernelnew.h:1642-1644) */
            if (safe && (L || R) && lh_max < ORC_SCALE_THR && t->ptn_invar[p] == 0.0) {
                for (j = 0; j < n; j++) o[c * n + j] = ldexp(o[c * n + j], ORC_SCALE_EXP);
                sd[c] += 1;
            }
        }
        if (!safe && (L || R) && lh_max < ORC_SCALE_THR && t->ptn_invar[p] == 0.0) {
            for (j = 0; j < blk; j++) o[j] = ldexp(o[j], ORC_SCALE_EXP);
            sd[0] += 1;
        }
    }
    t->partial_ops += 1;
    free(eL);
    free(eR);
    free(leafL);
    free(leafR);
}

/* computeTraversalInfo (phylotree.cpp:6031) + the packet loop: postorder recompute of every
 * stale directed branch in the subtree at `node` seen from `dad`. */
static void traverse(orc_tree *t, int dad, int node) {
    int d = dad * 3 + find_nei(t, dad, node);
    if (t->computed[d] || is_leaf(t, node)) return;
    for (int k = 0; k < t->deg[node]; k++) {
        int c = t->adj[node * 3 + k];
        if (c != dad) traverse(t, node, c);
    }
    compute_partial(t, dad, node);
    t->computed[d] = 1;
}

/* ---- branch log-likelihood (phylokernelnew.h:2658-3275) --------------------------- */

double orc_compute_likelihood_branch(orc_tree *t, int node, int dad, double *pattern_lh) {
    const int n = t->n, ncat = t->ncat, blk = t->block, P = t->nptn_pad;
    if (is_leaf(t, node)) {
        int tmp = node;
        node = dad;
        dad = tmp;
    }
    int kd = find_nei(t, dad, node), kn = find_nei(t, node, dad);
    traverse(t, dad, node);
    if (!is_leaf(t, dad)) traverse(t, node, dad);
    int d_dad = dad * 3 + kd, d_node = node * 3 + kn;
    double len = t->len[d_dad];
    double *val = (double *)malloc(sizeof(double) * blk);
    for (int c = 0; c < ncat; c++)
        for (int i = 0; i < n; i++)
            val[c * n + i] = exp(t->eval[i] * (t->rates[c] * len)) * t->props[c];
    double *plnode = NULL;
    if (is_leaf(t, dad)) {
        plnode = (double *)malloc(sizeof(double) * (t->unknown + 1) * blk);
        for (int s = 0; s <= t->unknown; s++)
            for (int c = 0; c < ncat; c++)
                for (int i = 0; i < n; i++)
                    plnode[s * blk + c * n + i] = val[c * n + i] * t->tip[s * n + i];
    }
    const double *pd = t->plh[d_dad];
    const uint16_t *sd = t->scl[d_dad];
    const double *pn = is_leaf(t, dad) ? NULL : t->plh[d_node];
    const uint16_t *sn = pn ? t->scl[d_node] : NULL;
    const uint8_t *st = is_leaf(t, dad) ? t->states + (size_t)dad * P : NULL;
    double tree_lh = 0.0;
    int p;
    for (p = 0; p < P; p++) {
        double lh_cat[64];
        double lh_ptn = 0.0;
        const double *a = pd + (size_t)p * blk;
        int c, i;
        for (c = 0; c < ncat; c++) {
            double acc = 0;
            if (pn) {
                const double *b = pn + (size_t)p * blk;
                for (i = 0; i < n; i++) acc += val[c * n + i] * b[c * n + i] * a[c * n + i];
            } else {
                const double *b = plnode + (size_t)st[p] * blk;
                for (i = 0; i < n; i++) acc += b[c * n + i] * a[c * n + i];
            }
            lh_cat[c] = acc;
        }
        double min_scale;
        if (t->safe) {
            int sum_s[64], ms;
            for (c = 0; c < ncat; c++)
                sum_s[c] = sd[(size_t)p * ncat + c] + (sn ? sn[(size_t)p * ncat + c] : 0);
            ms = sum_s[0];
            for (c = 1; c < ncat; c++)
                if (sum_s[c] < ms) ms = sum_s[c];
            for (c = 0; c < ncat; c++) {
                if (sum_s[c] == ms + 1) lh_cat[c] *= ORC_SCALE_THR;
                else if (sum_s[c] > ms + 1) lh_cat[c] = 0.0;
                lh_ptn += lh_cat[c];
            }
            min_scale = ms;
        } else {
            for (c = 0; c < ncat; c++) lh_ptn += lh_cat[c];
            min_scale = sd[p] + (sn ? sn[p] : 0);
        }
        lh_ptn = fabs(lh_ptn) + t->ptn_invar[p];
        double plh = log(lh_ptn) + min_scale * ORC_LOG_SCALE_THR;
        t->plh_out[p] = plh;
        if (p < t->nptn) tree_lh += plh * t->ptn_freq[p];
    }
    if (!isfinite(tree_lh)) {
        tree_lh = 0.0;
        for (p = 0; p < t->nptn; p++) {
            if (!isfinite(t->plh_out[p])) t->plh_out[p] = ORC_LOG_SCALE_THR * 4;
            tree_lh += t->plh_out[p] * t->ptn_freq[p];
        }
    }
    if (pattern_lh) memcpy(pattern_lh, t->plh_out, sizeof(double) * t->nptn);
    free(val);
    free(plnode);
    return tree_lh;
}

/* findFarthestLeaf (mtree.cpp:3040): height = longest path (edges) to a leaf below */
static int far_leaf(orc_tree *t, int node, int dad, int *height) {
    if (dad >= 0 && is_leaf(t, node)) {
        height[node] = 0;
        return node;
    }
    int res = -1;
    height[node] = 0;
    for (int k = 0; k < t->deg[node]; k++) {
        int c = t->adj[node * 3 + k];
        if (c == dad) continue;
        int leaf = far_leaf(t, c, node, height);
        if (height[node] < height[c] + 1) {
            height[node] = height[c] + 1;
            res = leaf;
        }
    }
    return res;
}

double orc_compute_likelihood(orc_tree *t, double *pattern_lh) {
    if (t->cur_u < 0) {
        int *h = (int *)calloc(t->nnode, sizeof(int));
        int leaf = far_leaf(t, 0, -1, h);
        free(h);
        t->cur_u = leaf;
        t->cur_k = 0;
    }
    int u = t->cur_u, v = t->adj[t->cur_u * 3 + t->cur_k];
    /* computeLikelihoodBranch(current_it, current_it_back->node): dad = u, node = v */
    return orc_compute_likelihood_branch(t, v, u, pattern_lh);
}

/* ---- theta + derivatives (phylokernelnew.h:2053-2650) ------------------------------ */

static void compute_theta(orc_tree *t, int d_dad, int d_node, int dad) {
    const int n = t->n, ncat = t->ncat, blk = t->block, P = t->nptn_pad;
    const double *pd = t->plh[d_dad];
    const uint16_t *sd = t->scl[d_dad];
    const double *pn = is_leaf(t, dad) ? NULL : t->plh[d_node];
    const uint16_t *sn = pn ? t->scl[d_node] : NULL;
    const uint8_t *st = pn ? NULL : t->states + (size_t)dad * P;
    for (int p = 0; p < P; p++) {
        double *th = t->theta + (size_t)p * blk;
        const double *a = pd + (size_t)p * blk;
        int c, i;
        if (pn) {
            const double *b = pn + (size_t)p * blk;
            for (i = 0; i < blk; i++) th[i] = b[i] * a[i];
        } else {
            const double *tp = t->tip + (size_t)st[p] * n;
            for (c = 0; c < ncat; c++)
                for (i = 0; i < n; i++) th[c * n + i] = tp[i] * a[c * n + i];
        }
        if (t->safe) {
            int ss[64], ms;
            for (c = 0; c < ncat; c++)
                ss[c] = sd[(size_t)p * ncat + c] + (sn ? sn[(size_t)p * ncat + c] : 0);
            ms = ss[0];
            for (c = 1; c < ncat; c++)
                if (ss[c] < ms) ms = ss[c];
            for (c = 0; c < ncat; c++) {
                if (ss[c] == ms + 1)
                    for (i = 0; i < n; i++) th[c * n + i] *= ORC_SCALE_THR;
                else if (ss[c] > ms + 1)
                    for (i = 0; i < n; i++) th[c * n + i] = 0.0;
            }
            t->scale_all[p] = (double)ms * ORC_LOG_SCALE_THR;
        } else {
            t->scale_all[p] = (double)(sd[p] + (sn ? sn[p] : 0)) * ORC_LOG_SCALE_THR;
        }
    }
}

void orc_compute_likelihood_derv(orc_tree *t, int node, int dad, double *df, double *ddf) {
    const int n = t->n, ncat = t->ncat, blk = t->block;
    if (is_leaf(t, node)) {
        int tmp = node;
        node = dad;
        dad = tmp;
    }
    int kd = find_nei(t, dad, node), kn = find_nei(t, node, dad);
    int d_dad = dad * 3 + kd, d_node = node * 3 + kn;
    if (!t->theta_computed) {
        traverse(t, dad, node);
        if (!is_leaf(t, dad)) traverse(t, node, dad);
        compute_theta(t, d_dad, d_node, dad);
        t->theta_computed = 1;
    }
    double len = t->len[d_dad];
    double *v0 = (double *)malloc(sizeof(double) * blk * 3);
    double *v1 = v0 + blk, *v2 = v1 + blk;
    for (int c = 0; c < ncat; c++)
        for (int i = 0; i < n; i++) {
            double cof = t->eval[i] * t->rates[c];
            double val = exp(cof * len) * t->props[c];
            double val1 = cof * val;
            v0[c * n + i] = val;
            v1[c * n + i] = val1;
            v2[c * n + i] = cof * val1;
        }
    double all_df = 0.0, all_ddf = 0.0;
    for (int p = 0; p < t->nptn_pad; p++) {
        const double *th = t->theta + (size_t)p * blk;
        double lh = 0, d1 = 0, d2 = 0;
        for (int i = 0; i < blk; i++) {
            lh += v0[i] * th[i];
            d1 += v1[i] * th[i];
            d2 += v2[i] * th[i];
        }
        lh = fabs(lh) + t->ptn_invar[p];
        if (p < t->nptn) {
            double inv = 1.0 / lh;
            double df_frac = d1 * inv, ddf_frac = d2 * inv;
            double fr = t->ptn_freq[p];
            double tmp1 = df_frac * fr, tmp2 = ddf_frac * fr;
            all_df += tmp1;
            all_ddf += tmp2 - tmp1 * df_frac;
            t->G[p] = df_frac;
        }
    }
    free(v0);
    if (!isfinite(all_df)) all_df = all_ddf = 0.0;
    *df = all_df;
    *ddf = all_ddf;
}

double orc_compute_likelihood_from_buffer(orc_tree *t) {
    const int n = t->n, ncat = t->ncat, blk = t->block;
    int u = t->cur_u, k = t->cur_k;
    double len = t->len[u * 3 + k];
    double *v0 = (double *)malloc(sizeof(double) * blk);
    for (int c = 0; c < ncat; c++)
        for (int i = 0; i < n; i++) {
            double cof = t->eval[i] * t->rates[c];
            v0[c * n + i] = exp(cof * len) * t->props[c];
        }
    double tree_lh = 0.0;
    for (int p = 0; p < t->nptn_pad; p++) {
        const double *th = t->theta + (size_t)p * blk;
        double lh = 0;
        for (int i = 0; i < blk; i++) lh += v0[i] * th[i];
        lh = fabs(lh) + t->ptn_invar[p];
        if (p < t->nptn) {
            double plh = log(fabs(lh)) + t->scale_all[p];
            t->plh_out[p] = plh;
            tree_lh += plh * t->ptn_freq[p];
        }
    }
    if (!isfinite(tree_lh)) {
        tree_lh = 0.0;
        for (int p = 0; p < t->nptn; p++) {
            if (!isfinite(t->plh_out[p])) t->plh_out[p] = ORC_LOG_SCALE_THR * 4;
            tree_lh += t->plh_out[p] * t->ptn_freq[p];
        }
    }
    free(v0);
    return tree_lh;
}

/* ---- Newton branch optimisation ----------------------------------------------------- */

/* computeFuncDerv (phylotree.cpp:2555): set length, derivatives of -lnL */
static void func_derv(orc_tree *t, double x, double *f, double *df) {
    int u = t->cur_u, v = t->adj[t->cur_u * 3 + t->cur_k];
    orc_set_length(t, u, v, x);
    double d1, d2;
    orc_compute_likelihood_derv(t, v, u, &d1, &d2);
    *f = -d1;
    *df = -d2;
    t->newton_evals++;
}

/* doNNI (tree/phylotree.cpp:4059-4125): neighbour entries (with their lengths and partials)
 * swap between u and v; central partials and those looking back at u or v are cleared. */
int orc_nni(orc_tree *t, int u, int v, int a, int b) {
    int ku_a = find_nei(t, u, a), kv_b = find_nei(t, v, b), ka_u = find_nei(t, a, u),
        kb_v = find_nei(t, b, v);
    if (is_leaf(t, u) || is_leaf(t, v) || find_nei(t, u, v) < 0 || ku_a < 0 || kv_b < 0)
        return -1;
    int du = u * 3 + ku_a, dv = v * 3 + kv_b, e;
    double *tp;
    uint16_t *ts;
    int ti;
    double tl;
    unsigned char tc;
    ti = t->adj[du]; t->adj[du] = t->adj[dv]; t->adj[dv] = ti;
    tl = t->len[du]; t->len[du] = t->len[dv]; t->len[dv] = tl;
    tp = t->plh[du]; t->plh[du] = t->plh[dv]; t->plh[dv] = tp;
    ts = t->scl[du]; t->scl[du] = t->scl[dv]; t->scl[dv] = ts;
    tc = t->computed[du]; t->computed[du] = t->computed[dv]; t->computed[dv] = tc;
    t->adj[a * 3 + ka_u] = v;
    t->adj[b * 3 + kb_v] = u;
    t->computed[u * 3 + find_nei(t, u, v)] = 0;
    t->computed[v * 3 + find_nei(t, v, u)] = 0;
    clear_reverse(t, v, u);
    clear_reverse(t, u, v);
    for (e = 0; e < t->nedges; e++) {
        if ((t->eu[e] == u && t->ev[e] == a) || (t->eu[e] == a && t->ev[e] == u)) {
            t->eu[e] = v;
            t->ev[e] = a;
        } else if ((t->eu[e] == v && t->ev[e] == b) || (t->eu[e] == b && t->ev[e] == v)) {
            t->eu[e] = u;
            t->ev[e] = b;
        }
    }
    t->theta_computed = 0;
    t->cur_u = -1;
    return 0;
}

/* marks the nodes of the subtree at v (away from u) */
static void mark_subtree(const orc_tree *t, int v, int u, unsigned char *m) {
    m[v] = 1;
    for (int k = 0; k < t->deg[v]; k++)
        if (t->adj[v * 3 + k] != u) mark_subtree(t, t->adj[v * 3 + k], v, m);
}

/* clears every partial whose subtree holds node x (the directed branches pointing at x) */
static void clear_toward(orc_tree *t, int x) {
    for (int k = 0; k < t->deg[x]; k++) {
        int c = t->adj[x * 3 + k];
        t->computed[c * 3 + find_nei(t, c, x)] = 0;
        clear_reverse(t, c, x);
    }
}

/* SPR move with the geometry of assessSPRMove (tree/phylotree.cpp:4822-4880): the subtree at
 * `node` is pruned from `dad` (internal), whose two other neighbours s1 < s2 (by node id; the
 * reference takes them in its neighbour order) are joined by one branch of their summed length;
 * dad is then inserted into the branch (node2, dad2), its entry that pointed at s1 taking dad2
 * and the one that pointed at s2 node2, each half the branch's length.  Edges: (dad, s1) becomes (s1, s2), (dad, s2) becomes (dad, dad2),
 * (node2, dad2) becomes (dad, node2).  The four neighbour entries that keep their subtree keep
 * their partials ((s1->s2) takes (dad->s2)'s, (s2->s1) (dad->s1)'s, (dad->dad2) (node2->dad2)'s,
 * (dad->node2) (dad2->node2)'s); every partial whose subtree holds dad before or after the move
 * is cleared, which also covers any of the four whose subtree did change. */
int orc_spr(orc_tree *t, int node, int dad, int node2, int dad2) {
    if (node < 0 || dad < 0 || node2 < 0 || dad2 < 0 || node >= t->nnode || dad >= t->nnode ||
        node2 >= t->nnode || dad2 >= t->nnode)
        return -1;
    int kn = find_nei(t, dad, node);
    if (is_leaf(t, dad) || kn < 0 || find_nei(t, node2, dad2) < 0 || node2 == dad || dad2 == dad)
        return -1;
    unsigned char *in_s = calloc((size_t)t->nnode, 1);
    mark_subtree(t, node, dad, in_s);
    int bad = in_s[node2] || in_s[dad2];
    free(in_s);
    if (bad) return -1;
    int ks[2], nk = 0;
    for (int k = 0; k < 3; k++)
        if (k != kn) ks[nk++] = k;
    if (t->adj[dad * 3 + ks[0]] > t->adj[dad * 3 + ks[1]]) {
        int tk = ks[0];
        ks[0] = ks[1];
        ks[1] = tk;
    }
    int s1 = t->adj[dad * 3 + ks[0]], s2 = t->adj[dad * 3 + ks[1]];
    int ia = dad * 3 + ks[0], ib = dad * 3 + ks[1];
    int ic = s1 * 3 + find_nei(t, s1, dad), id = s2 * 3 + find_nei(t, s2, dad);
    int ie = node2 * 3 + find_nei(t, node2, dad2), iff = dad2 * 3 + find_nei(t, dad2, node2);
    double l1 = t->len[ia], l2 = t->len[ib], l = t->len[ie];
    clear_toward(t, dad);
    int idx[6] = {ic, id, ia, ib, ie, iff}, src[6] = {ib, ia, ie, iff, ic, id};
    double *pl[6];
    uint16_t *sc[6];
    unsigned char cm[6];
    for (int i = 0; i < 6; i++) {
        pl[i] = t->plh[src[i]];
        sc[i] = t->scl[src[i]];
        cm[i] = t->computed[src[i]];
    }
    t->adj[ic] = s2;
    t->adj[id] = s1;
    t->len[ic] = t->len[id] = l1 + l2;
    t->adj[ia] = dad2;
    t->adj[ib] = node2;
    t->adj[ie] = dad;
    t->adj[iff] = dad;
    t->len[ia] = t->len[ib] = t->len[ie] = t->len[iff] = l / 2;
    for (int i = 0; i < 6; i++) {
        t->plh[idx[i]] = pl[i];
        t->scl[idx[i]] = sc[i];
        t->computed[idx[i]] = cm[i];
    }
    clear_toward(t, dad);
    int e_s1 = -1, e_s2 = -1, e_r = -1;
    for (int e = 0; e < t->nedges; e++) {
        int a = t->eu[e], b = t->ev[e];
        if ((a == dad && b == s1) || (a == s1 && b == dad)) e_s1 = e;
        else if ((a == dad && b == s2) || (a == s2 && b == dad)) e_s2 = e;
        else if ((a == node2 && b == dad2) || (a == dad2 && b == node2)) e_r = e;
    }
    t->eu[e_s1] = s1;
    t->ev[e_s1] = s2;
    t->eu[e_s2] = dad;
    t->ev[e_s2] = dad2;
    t->eu[e_r] = dad;
    t->ev[e_r] = node2;
    t->theta_computed = 0;
    t->cur_u = -1;
    return 0;
}

void orc_compute_func_derv(orc_tree *t, int node1, int node2, double value, int new_branch,
                           double *f, double *df) {
    t->cur_u = node1;
    t->cur_k = find_nei(t, node1, node2);
    if (new_branch) t->theta_computed = 0;
    func_derv(t, value, f, df);
}

/* minimizeNewton (utils/optimization.cpp:422-499) */
static double minimize_newton(orc_tree *t, double x1, double xguess, double x2, double xacc,
                              int maxstep) {
    double df, dx, f, temp, xh, xl, rts, rts_old;
    int j;
    rts = xguess;
    if (rts < x1) rts = x1;
    if (rts > x2) rts = x2;
    func_derv(t, rts, &f, &df);
    if (!isfinite(f) || !isfinite(df)) return rts;
    if (df >= 0.0 && fabs(f) < xacc) return rts;
    if (f < 0.0) {
        xl = rts;
        xh = x2;
    } else {
        xh = rts;
        xl = x1;
    }
    dx = fabs(xh - xl);
    for (j = 1; j <= maxstep; j++) {
        rts_old = rts;
        if ((df <= 0.0) || (((rts - xh) * df - f) * ((rts - xl) * df - f) >= 0.0)) {
            dx = 0.5 * (xh - xl);
            rts = xl + dx;
            if (xl == rts) return rts;
        } else {
            dx = f / df;
            temp = rts;
            rts -= dx;
            if (temp == rts) return rts;
        }
        if (fabs(dx) < xacc || (j == maxstep)) return rts_old;
        func_derv(t, rts, &f, &df);
        if (!isfinite(f) || !isfinite(df)) return rts;
        if (df > 0.0 && fabs(f) < xacc) return rts;
        if (f < 0.0) xl = rts;
        else if (f > 0.0) xh = rts;
    }
    return 0.0;
}

void orc_optimize_one_branch(orc_tree *t, int node1, int node2, int clear_lh, int max_nr_step) {
    if (node1 < 0 || node1 >= t->nnode || node2 < 0 || node2 >= t->nnode) return;
    int k = find_nei(t, node1, node2);
    if (k < 0) return;
    t->cur_u = node1;
    t->cur_k = k;
    double cur = t->len[node1 * 3 + k];
    t->theta_computed = 0;
    t->newton_evals = 0;
    double optx = minimize_newton(t, t->min_bl, cur, t->max_bl, t->min_bl, max_nr_step);
    if (optx > t->max_bl * 0.95) {
        double opt_lh = orc_compute_likelihood_from_buffer(t);
        orc_set_length(t, node1, node2, cur);
        double orig_lh = orc_compute_likelihood_from_buffer(t);
        if (orig_lh > opt_lh) optx = cur;
    }
    orc_set_length(t, node1, node2, optx);
    if (clear_lh && cur != optx) {
        clear_reverse(t, node1, node2);
        clear_reverse(t, node2, node1);
    }
}

/* getPreOrderBranches (mtree.cpp:3062): neighbours visited by ascending height, using the
 * reference's pairwise-swap ordering */
static void preorder_branches(orc_tree *t, int node, int dad, const int *height, int *n1,
                              int *n2, int *cnt) {
    if (dad >= 0) {
        n1[*cnt] = node;
        n2[*cnt] = dad;
        (*cnt)++;
    }
    int nv[3], nd = t->deg[node], i, j;
    for (i = 0; i < nd; i++) nv[i] = t->adj[node * 3 + i];
    for (i = 0; i < nd; i++)
        for (j = i + 1; j < nd; j++)
            if (height[nv[i]] > height[nv[j]]) {
                int tmp = nv[i];
                nv[i] = nv[j];
                nv[j] = tmp;
            }
    for (i = 0; i < nd; i++)
        if (nv[i] != dad) preorder_branches(t, nv[i], node, height, n1, n2, cnt);
}

double orc_optimize_all_branches(orc_tree *t, int iterations, double tolerance, int max_nr_step) {
    int *h = (int *)calloc(t->nnode, sizeof(int));
    int far = far_leaf(t, 0, -1, h);
    far_leaf(t, far, -1, h);
    int *n1 = (int *)malloc(sizeof(int) * t->nnode), *n2 = (int *)malloc(sizeof(int) * t->nnode);
    int cnt = 0;
    preorder_branches(t, far, -1, h, n1, n2, &cnt);
    free(h);
    /* computeLikelihoodBranch(nodes[0]->findNeighbor(nodes2[0]), nodes[0]) */
    double tree_lh = orc_compute_likelihood_branch(t, n2[0], n1[0], NULL);
    double *saved = (double *)malloc(sizeof(double) * t->nedges);
    for (int it = 0; it < iterations; it++) {
        orc_get_lengths(t, saved);
        for (int j = 0; j < cnt; j++) orc_optimize_one_branch(t, n1[j], n2[j], 1, max_nr_step);
        double new_lh = orc_compute_likelihood_from_buffer(t);
        if (new_lh < tree_lh - tolerance * 0.1) {
            orc_clear_all_partial_lh(t);
            for (int e = 0; e < t->nedges; e++) orc_set_length(t, t->eu[e], t->ev[e], saved[e]);
            new_lh = orc_compute_likelihood(t, NULL);
            free(saved);
            free(n1);
            free(n2);
            return new_lh;
        }
        if (tree_lh <= new_lh && new_lh <= tree_lh + tolerance) {
            tree_lh = new_lh;
            break;
        }
        tree_lh = new_lh;
    }
    free(saved);
    free(n1);
    free(n2);
    return tree_lh;
}

/* ---- inspection ---------------------------------------------------------------------- */

int orc_get_partial(orc_tree *t, int node, int dad, double *partial, uint16_t *scale) {
    int k = find_nei(t, dad, node);
    if (k < 0) return -1;
    int d = dad * 3 + k;
    if (!t->plh[d] || !t->computed[d]) return -2;
    if (partial) memcpy(partial, t->plh[d], sizeof(double) * (size_t)t->nptn_pad * t->block);
    if (scale)
        memcpy(scale, t->scl[d], 2 * (size_t)t->nptn_pad * (t->safe ? t->ncat : 1));
    return 0;
}

int orc_get_theta(orc_tree *t, double *theta, double *scale_all) {
    if (!t->theta_computed) return -1;
    if (theta) memcpy(theta, t->theta, sizeof(double) * (size_t)t->nptn_pad * t->block);
    if (scale_all) memcpy(scale_all, t->scale_all, sizeof(double) * t->nptn_pad);
    return 0;
}

int orc_get_df_frac(orc_tree *t, double *out) {
    memcpy(out, t->G, sizeof(double) * t->nptn);
    return 0;
}

int orc_nptn_pad(orc_tree *t) { return t->nptn_pad; }
long long orc_partial_ops(orc_tree *t) { return t->partial_ops; }
int orc_last_newton_evals(orc_tree *t) { return t->newton_evals; }
