/*
 * synth.c -- seeded synthetic workload generator (host C, no GPU).
 *
 * Produces the inputs the likelihood path runs on: a random unrooted binary tree with
 * exponential branch lengths, sequences simulated down that tree under a reversible
 * substitution model with discrete rate categories, optional gap cells (all-ones tip code),
 * and the pattern compression of the alignment into unique columns with integer weights.
 *
 * Deterministic for a given seed (xoshiro256** streams seeded through splitmix64), so the
 * same case can be regenerated on any host.  Used by bench.py and the tests to build inputs;
 * it computes no likelihoods.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    uint64_t s[4];
} rng_t;

static uint64_t splitmix64(uint64_t *x) {
    uint64_t z = (*x += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
static void rng_seed(rng_t *r, uint64_t seed) {
    uint64_t x = seed;
    for (int i = 0; i < 4; i++) r->s[i] = splitmix64(&x);
}
static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
static inline uint64_t rng_next(rng_t *r) {
    uint64_t *s = r->s;
    uint64_t res = rotl(s[1] * 5, 7) * 9;
    uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return res;
}
static inline double rng_unif(rng_t *r) { return (rng_next(r) >> 11) * 0x1.0p-53; }

/* Random unrooted binary tree by stepwise addition of leaves onto uniformly chosen edges.
 * Leaves 0..ntaxa-1, internal nodes ntaxa..2*ntaxa-3; 2*ntaxa-3 edges.  Lengths ~ Exp(mean),
 * floored at 1e-6.  Returns the number of edges, or -1 when ntaxa < 3. */
int gems_synth_tree(int ntaxa, double mean_len, uint64_t seed, int *eu, int *ev, double *len) {
    if (ntaxa < 3) return -1;
    rng_t r;
    rng_seed(&r, seed);
    int ne = 0, next_internal = ntaxa;
    int c = next_internal++;
    for (int i = 0; i < 3; i++) {
        eu[ne] = c;
        ev[ne] = i;
        ne++;
    }
    for (int leaf = 3; leaf < ntaxa; leaf++) {
        int e = (int)(rng_unif(&r) * ne);
        if (e >= ne) e = ne - 1;
        int u = eu[e], v = ev[e];
        int m = next_internal++;
        eu[e] = u;
        ev[e] = m;
        eu[ne] = m;
        ev[ne] = v;
        ne++;
        eu[ne] = m;
        ev[ne] = leaf;
        ne++;
    }
    for (int e = 0; e < ne; e++) {
        double x = -mean_len * log(1.0 - rng_unif(&r));
        len[e] = x < 1e-6 ? 1e-6 : x;
    }
    return ne;
}

/* Transition matrix P(t) = evec * diag(exp(eval*t)) * inv_evec, rows clamped at 0 and
 * renormalised, stored as cumulative rows for sampling. */
static void cum_pmatrix(int n, const double *eval, const double *evec, const double *inv_evec,
                        double t, double *cum) {
    double *ex = (double *)malloc(sizeof(double) * n);
    for (int i = 0; i < n; i++) ex[i] = exp(eval[i] * t);
    for (int x = 0; x < n; x++) {
        double s = 0;
        for (int y = 0; y < n; y++) {
            double a = 0;
            for (int i = 0; i < n; i++) a += evec[x * n + i] * ex[i] * inv_evec[i * n + y];
            if (a < 0) a = 0;
            cum[x * n + y] = a;
            s += a;
        }
        double acc = 0;
        for (int y = 0; y < n; y++) {
            acc += cum[x * n + y] / s;
            cum[x * n + y] = acc;
        }
        cum[x * n + n - 1] = 1.0;
    }
    free(ex);
}

static inline int sample_cum(const double *cum, int n, double u) {
    int y = 0;
    while (y < n - 1 && u >= cum[y]) y++;
    return y;
}

/* Simulate nsites sites down the tree.  The root is internal node ntaxa; root states ~ freq;
 * each site draws a rate category from props.  out is [ntaxa][nsites] state bytes.
 * A fraction gap_frac of the cells is replaced by gap_state (the all-ones tip code).
 * Returns 0 on success. */
int gems_synth_simulate(int ntaxa, int nedges, const int *eu, const int *ev, const double *len,
                        int n, int ncat, const double *rates, const double *props,
                        const double *eval, const double *evec, const double *inv_evec,
                        const double *freq, long long nsites, double gap_frac, int gap_state,
                        uint64_t seed, uint8_t *out) {
    int nnode = nedges + 1;
    /* adjacency */
    int *deg = (int *)calloc(nnode, sizeof(int));
    int *adj = (int *)malloc(sizeof(int) * nnode * 3);
    double *alen = (double *)malloc(sizeof(double) * nnode * 3);
    for (int e = 0; e < nedges; e++) {
        int u = eu[e], v = ev[e];
        if (deg[u] >= 3 || deg[v] >= 3) {
            free(deg);
            free(adj);
            free(alen);
            return -1;
        }
        adj[u * 3 + deg[u]] = v;
        alen[u * 3 + deg[u]++] = len[e];
        adj[v * 3 + deg[v]] = u;
        alen[v * 3 + deg[v]++] = len[e];
    }
    /* preorder from root (internal node ntaxa, or node 0 for tiny trees) */
    int root = nnode > ntaxa ? ntaxa : 0;
    int *order = (int *)malloc(sizeof(int) * nnode), *parent = (int *)malloc(sizeof(int) * nnode);
    double *plen = (double *)malloc(sizeof(double) * nnode);
    int head = 0, tail = 0;
    order[tail++] = root;
    parent[root] = -1;
    plen[root] = 0;
    while (head < tail) {
        int u = order[head++];
        for (int k = 0; k < deg[u]; k++) {
            int v = adj[u * 3 + k];
            if (v == parent[u]) continue;
            parent[v] = u;
            plen[v] = alen[u * 3 + k];
            order[tail++] = v;
        }
    }
    double *cum = (double *)malloc(sizeof(double) * (size_t)nnode * ncat * n * n);
    for (int v = 0; v < nnode; v++) {
        if (parent[v] < 0) continue;
        for (int c = 0; c < ncat; c++)
            cum_pmatrix(n, eval, evec, inv_evec, rates[c] * plen[v],
                        cum + ((size_t)v * ncat + c) * n * n);
    }
    double *fcum = (double *)malloc(sizeof(double) * n);
    double *ccum = (double *)malloc(sizeof(double) * ncat);
    double acc = 0, fs = 0, ps = 0;
    for (int i = 0; i < n; i++) fs += freq[i];
    for (int i = 0; i < n; i++) {
        acc += freq[i] / fs;
        fcum[i] = acc;
    }
    fcum[n - 1] = 1.0;
    acc = 0;
    for (int c = 0; c < ncat; c++) ps += props[c];
    for (int c = 0; c < ncat; c++) {
        acc += props[c] / ps;
        ccum[c] = acc;
    }
    ccum[ncat - 1] = 1.0;

    /* sites are simulated in chunks so that each chunk has its own stream (reproducible and
     * independent of threading) */
    const long long CH = 4096;
    long long nchunk = (nsites + CH - 1) / CH;
#pragma omp parallel for schedule(dynamic, 4)
    for (long long ch = 0; ch < nchunk; ch++) {
        rng_t r;
        rng_seed(&r, seed * 0x100000001B3ULL + (uint64_t)ch + 1);
        long long s0 = ch * CH, s1 = s0 + CH < nsites ? s0 + CH : nsites;
        uint8_t *st = (uint8_t *)malloc(nnode);
        for (long long s = s0; s < s1; s++) {
            int cat = sample_cum(ccum, ncat, rng_unif(&r));
            st[root] = (uint8_t)sample_cum(fcum, n, rng_unif(&r));
            for (int k = 1; k < nnode; k++) {
                int v = order[k];
                const double *cm = cum + (((size_t)v * ncat + cat) * n + st[parent[v]]) * n;
                st[v] = (uint8_t)sample_cum(cm, n, rng_unif(&r));
            }
            for (int t = 0; t < ntaxa; t++) {
                uint8_t x = st[t];
                if (gap_frac > 0 && rng_unif(&r) < gap_frac) x = (uint8_t)gap_state;
                out[(size_t)t * nsites + s] = x;
            }
        }
        free(st);
    }
    free(fcum);
    free(ccum);
    free(cum);
    free(order);
    free(parent);
    free(plen);
    free(deg);
    free(adj);
    free(alen);
    return 0;
}

/* Pattern compression: unique alignment columns in order of first appearance with their
 * counts.  aln is [ntaxa][nsites]; pat receives [ntaxa][npat] (caller provides room for
 * nsites columns), weights[npat].  Returns npat. */
long long gems_synth_compress(int ntaxa, long long nsites, const uint8_t *aln, uint8_t *pat,
                              double *weights) {
    uint64_t cap = 1;
    while (cap < (uint64_t)nsites * 2) cap <<= 1;
    long long *table = (long long *)malloc(sizeof(long long) * cap);
    for (uint64_t i = 0; i < cap; i++) table[i] = -1;
    uint64_t *hash = (uint64_t *)malloc(sizeof(uint64_t) * nsites);
    /* column hashes (FNV-1a over the column bytes) */
#pragma omp parallel for schedule(static)
    for (long long s = 0; s < nsites; s++) {
        uint64_t h = 1469598103934665603ULL;
        for (int t = 0; t < ntaxa; t++) {
            h ^= aln[(size_t)t * nsites + s];
            h *= 1099511628211ULL;
        }
        hash[s] = h;
    }
    long long *first = (long long *)malloc(sizeof(long long) * nsites); /* pattern -> column */
    long long npat = 0;
    for (long long s = 0; s < nsites; s++) {
        uint64_t h = hash[s];
        uint64_t slot = h & (cap - 1);
        for (;;) {
            long long p = table[slot];
            if (p < 0) {
                table[slot] = npat;
                first[npat] = s;
                weights[npat] = 1.0;
                npat++;
                break;
            }
            long long s2 = first[p];
            if (hash[s2] == h) {
                int same = 1;
                for (int t = 0; t < ntaxa; t++)
                    if (aln[(size_t)t * nsites + s] != aln[(size_t)t * nsites + s2]) {
                        same = 0;
                        break;
                    }
                if (same) {
                    weights[p] += 1.0;
                    break;
                }
            }
            slot = (slot + 1) & (cap - 1);
        }
    }
#pragma omp parallel for schedule(static)
    for (int t = 0; t < ntaxa; t++)
        for (long long p = 0; p < npat; p++)
            pat[(size_t)t * npat + p] = aln[(size_t)t * nsites + first[p]];
    free(first);
    free(hash);
    free(table);
    return npat;
}
