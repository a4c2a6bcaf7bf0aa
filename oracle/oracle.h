/*
 * oracle.h -- FP64 CPU restatement of IQ-TREE's reversible Felsenstein likelihood path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path in gems_b200:
 * only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may load it.
 * The product never calls it, and nothing here runs on a GPU.
 *
 * Each function names the reference file:line whose behaviour it restates (paths are
 * relative to the IQ-TREE 3 source tree).  The arithmetic follows the reference formulas
 * (eigen-space partials, 2^-256 underflow scaling with uint16 counters, NORM and SAFE modes,
 * pattern-weighted lnL and derivative sums, safeguarded Newton) in plain scalar loops.
 */
#ifndef GEMS_ORACLE_H
#define GEMS_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_tree orc_tree;

/* ---- model setup (tree/ + model/ + utils/ restatements) ---- */

/* Discrete-Gamma category rates, mean (cut_median=0) or median (cut_median=1) method.
 * model/rategamma.cpp:98-172 (computeRates / computeRatesMean) with the PAML helpers
 * cmpLnGamma :305, cmpIncompleteGamma :325, cmpPointNormal :389, cmpPointChi2 :420. */
void orc_gamma_rates(double alpha, int ncat, int cut_median, double *rates);

/* Reversible eigensystem from exchangeabilities (upper triangle, row-major, n(n-1)/2 entries)
 * and state frequencies, normalised to total_num_subst=1.
 * utils/eigendecomposition.cpp:165 eigensystem_sym, :478 computeRateMatrix, :521 eliminateZero,
 * :557 symmetrizeRateMatrix, :581 tred2, :667 tqli.  Returns 0 on success. */
int orc_eigensystem_sym(int n, const double *rates_upper, const double *freq,
                        double *eval, double *evec, double *inv_evec);

/* ---- tree session ---- */

/* Build an unrooted tree.  Leaves are nodes 0..ntaxa-1 (taxon id == row of the tip matrix),
 * internal nodes ntaxa..nnode-1.  Each node's neighbour list is filled in edge order.
 * safe != 0 selects SAFE_NUMERIC (per-category scaling), else NORM.
 * phylotree.cpp:905-1213 (initializeAllPartialLh, per-directed-branch buffers). */
orc_tree *orc_tree_new(int ntaxa, int nedges, const int *eu, const int *ev, const double *elen,
                       int nstates, int ncat, int safe);
void orc_tree_free(orc_tree *t);

/* eval[n], evec[n*n], inv_evec[n*n] row-major; rates[ncat], props[ncat]; state_freq[n]. */
void orc_set_model(orc_tree *t, const double *eval, const double *evec, const double *inv_evec,
                   const double *rates, const double *props, double p_invar,
                   const double *state_freq);

/* states[ntaxa][nptn] converted state bytes; freq[nptn] pattern weights;
 * const_char[nptn] (constant state of the pattern, or >STATE_UNKNOWN when variable; may be
 * NULL when p_invar == 0).  phylotreesse.cpp:537 computePtnFreq, :549 computePtnInvar. */
void orc_set_patterns(orc_tree *t, int nptn, const uint8_t *states, const double *freq,
                      const uint8_t *const_char);

void orc_set_branch_limits(orc_tree *t, double min_bl, double max_bl);
int orc_set_length(orc_tree *t, int u, int v, double len);
double orc_get_length(orc_tree *t, int u, int v);
/* lengths in the constructor's edge order */
void orc_get_lengths(orc_tree *t, double *out);

/* phylotree.cpp:680 clearAllPartialLH */
void orc_clear_all_partial_lh(orc_tree *t);

/* phylotree.cpp:1258 computeLikelihood (pattern_lh may be NULL). */
double orc_compute_likelihood(orc_tree *t, double *pattern_lh);
/* phylotreesse.cpp:216 computeLikelihoodBranch(dad->findNeighbor(node), dad) */
double orc_compute_likelihood_branch(orc_tree *t, int node, int dad, double *pattern_lh);
/* phylotreesse.cpp:221 computeLikelihoodDerv(dad->findNeighbor(node), dad) */
void orc_compute_likelihood_derv(orc_tree *t, int node, int dad, double *df, double *ddf);
/* phylotreesse.cpp:226 computeLikelihoodFromBuffer (current_it, theta resident) */
double orc_compute_likelihood_from_buffer(orc_tree *t);
/* phylotree.cpp:4059 doNNI: swap subtree a (at u) with subtree b (at v) across branch (u, v) */
int orc_nni(orc_tree *t, int u, int v, int a, int b);
/* phylotree.cpp:4822 assessSPRMove's move: prune the subtree at node from dad, regraft dad into
 * the branch (node2, dad2) (halves of its length; dad's other branches joined, lengths summed) */
int orc_spr(orc_tree *t, int node, int dad, int node2, int dad2);
/* phylotree.cpp:2555 computeFuncDerv on branch (node1, node2) at length value: f = -dlnL/dt,
 * df = -d2lnL/dt2, theta rebuilt first when new_branch != 0 */
void orc_compute_func_derv(orc_tree *t, int node1, int node2, double value, int new_branch,
                           double *f, double *df);
/* phylotree.cpp:2620 optimizeOneBranch */
void orc_optimize_one_branch(orc_tree *t, int node1, int node2, int clear_lh, int max_nr_step);
/* phylotree.cpp:2724 optimizeAllBranches(my_iterations, tolerance, maxNRStep) */
double orc_optimize_all_branches(orc_tree *t, int iterations, double tolerance, int max_nr_step);

/* Inspection: partial (nptn_pad*block doubles) and scale counts of directed branch dad->node
 * (uint16 [nptn_pad] NORM or [nptn_pad*ncat] SAFE).  Returns 0 if the buffer is valid. */
int orc_get_partial(orc_tree *t, int node, int dad, double *partial, uint16_t *scale);
/* theta_all (nptn_pad*block) and buffer_scale_all (nptn_pad) of the current branch */
int orc_get_theta(orc_tree *t, double *theta, double *scale_all);
/* G_matrix row (df_frac per pattern) written by the last derivative call */
int orc_get_df_frac(orc_tree *t, double *out);
int orc_nptn_pad(orc_tree *t);
/* number of internal partial updates executed since creation (site-partial updates / nptn) */
long long orc_partial_ops(orc_tree *t);
/* Newton iteration count of the last optimize_one_branch (computeFuncDerv calls) */
int orc_last_newton_evals(orc_tree *t);
void orc_set_threads(int nthreads);

#ifdef __cplusplus
}
#endif
#endif
