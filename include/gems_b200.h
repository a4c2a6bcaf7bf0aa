/*
 * gems_b200.h -- C-ABI of the B200 (sm_100a) Felsenstein likelihood kernels.
 *
 * Two layers, both plain C (pointers, sizes, int status codes; no CUDA or torch types):
 *
 *  1. Kernel set ("gems_*"): what a new LikelihoodKernel value of IQ-TREE's PhyloTree
 *     forwards its member-function pointers to.  The device session owns every partial
 *     likelihood buffer, scale counter, theta buffer and tip byte; the caller keeps topology
 *     and cache flags and names buffers by slot id.  Replaces the pointer targets that
 *     PhyloTree::setLikelihoodKernel installs (tree/phylotreesse.cpp:91-199):
 *        computePartialLikelihoodPointer   (tree/phylotree.h:902-903)   -> gems_compute_partial
 *                                        (one entry, one packet; gems_traverse: the whole list)
 *        computeLikelihoodBranchPointer    (tree/phylotree.h:948-950)   -> gems_branch_lnl
 *        computeLikelihoodDervPointer      (tree/phylotree.h:1343-1345) -> gems_branch_derv
 *        computeLikelihoodFromBufferPointer(tree/phylotree.h:1002-1003) -> gems_lnl_from_buffer
 *     plus the Newton loop of PhyloTree::optimizeOneBranch (tree/phylotree.cpp:2620-2670,
 *     utils/optimization.cpp:422-499) -> gems_newton_branch.
 *
 *  2. Tree mirror ("gems_tree_*"): a C++ re-statement of the PhyloTree calls on the path
 *     (computeLikelihood, computeLikelihoodBranch, computeLikelihoodDerv,
 *     computeLikelihoodFromBuffer, optimizeOneBranch, optimizeAllBranches, clearAllPartialLH)
 *     driving layer 1, for callers that do not bring their own PhyloTree.
 *
 * Every call returns a gems_status.  Nothing exits the process; the reference's outError /
 * ASSERT paths map onto these codes.  Calls on one session are not thread-safe; distinct
 * sessions may be used from distinct threads (each session owns one CUDA stream).
 */
#ifndef GEMS_B200_H
#define GEMS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    GEMS_OK = 0,
    GEMS_ERR_OOM = 1,               /* device allocation failed */
    GEMS_ERR_ADMISSION = 2,         /* footprint exceeds the admission budget */
    GEMS_ERR_NUMERIC_UNDERFLOW = 3, /* non-finite derivative (reference: "-safe" advice) */
    GEMS_ERR_TIMEOUT = 4,           /* a bounded device wait ran out */
    GEMS_ERR_BAD_ARG = 5,
    GEMS_ERR_CUDA = 6,              /* CUDA runtime error (message in gems_last_error) */
    GEMS_ERR_STATE = 7,             /* call out of order (e.g. no model, theta not computed) */
    GEMS_ERR_NO_DEVICE = 8
} gems_status;

enum { GEMS_PREC_FP64 = 0, GEMS_PREC_MIXED = 1 };
enum { GEMS_SCALE_NORM = 0, GEMS_SCALE_SAFE = 1 };
enum { GEMS_CHILD_TIP = 0, GEMS_CHILD_PARTIAL = 1 };

typedef struct gems_session gems_session;

typedef struct {
    int ntaxa;      /* leaves; tip rows 0..ntaxa-1 */
    int nptn;       /* unique patterns (aln->size()) */
    int nstates;    /* 4 (DNA), 20 (protein), 61 (codon) or any 2..64 */
    int ncat;       /* rate categories, 1..16 (ncat_mix of the reference) */
    int nslots;     /* partial-likelihood buffers the session allocates */
    int precision;  /* GEMS_PREC_FP64 or GEMS_PREC_MIXED */
    int scaling;    /* GEMS_SCALE_NORM or GEMS_SCALE_SAFE (reference SAFE_NUMERIC) */
    int device;     /* CUDA device ordinal */
} gems_session_desc;

/* One node of a traversal: recompute the partial of slot dst from two children.
 * Mirrors TraversalInfo (tree/phylotree.h) for a binary node: the children are
 * (kind, id): GEMS_CHILD_TIP with a taxon id, or GEMS_CHILD_PARTIAL with a slot id;
 * len_* is the branch length from the node to that child. */
typedef struct {
    int dst_slot;
    int left_kind, left_id;
    int right_kind, right_id;
    int pad_;
    double left_len, right_len;
} gems_op;

/* A branch for lnL / derivatives: dad side is always a partial slot ("dad_branch" partial);
 * node side is a tip or a partial slot.  length is the branch length. */
typedef struct {
    int dad_slot;
    int node_kind, node_id;
    int pad_;
    double length;
} gems_branch;

/* ---- session ---- */
const char *gems_version(void);
const char *gems_last_error(void);
int gems_device_count(int *count);
/* Bytes a session with this descriptor holds on the device (admission by footprint). */
int gems_session_footprint(const gems_session_desc *desc, size_t *bytes);
int gems_session_create(const gems_session_desc *desc, gems_session **out);
int gems_session_destroy(gems_session *s);
int gems_session_sync(gems_session *s);
/* the descriptor the session was created with */
int gems_session_info(gems_session *s, gems_session_desc *desc);
/* the CUDA stream (cudaStream_t) the session launches on, for event timing by the caller */
int gems_session_stream(gems_session *s, void **stream);
/* Session options.  GEMS_OPT_TENSOR_CORES (default 1): the mixed-precision 20-state traversal
 * runs on tcgen05 split-TF32 products; 0 selects the FP32 CUDA-core kernel.
 * GEMS_OPT_TILED_FP64 (default 1): the FP64 61-state traversal (1 to 8 categories) runs as
 * register-tiled GEMMs over 128-row tiles; 0 selects the per-row kernel (same values, bit for
 * bit). */
enum { GEMS_OPT_TENSOR_CORES = 1, GEMS_OPT_TILED_FP64 = 2, GEMS_OPT_AUTOTUNE = 3,
       GEMS_OPT_NEWTON_SHARE = 4, GEMS_OPT_TC20_HALVES = 5, GEMS_OPT_TC61_ROLES = 6 };
/* GEMS_OPT_TC61_ROLES (default 1): the tcgen05 61-state traversal gives the parts of a step to
 * different warps (operand split, MMA issue, epilogue, copies) working on consecutive steps at
 * once, with double-buffered accumulators; 0 selects the form in which every warp runs the
 * parts one after the other.  The values are the same bits either way. */
/* GEMS_OPT_TC20_HALVES (default 0): the tcgen05 20-state traversal runs two CTAs per SM, each
 * taking its tile two categories at a time with every internal child copied back from the
 * slot (no forwarding), instead of one CTA per SM with all categories at once; the values are
 * the same bits either way. */
/* GEMS_OPT_NEWTON_SHARE (default 1): the device Newton loop (gems_newton_branch) is one
 * cooperative kernel whose blocks are all resident at once; with value k it takes at most 1/k
 * of the GPU's resident blocks, so that it runs beside other sessions' work instead of waiting
 * for the whole GPU (a server with many sessions sets k > 1).  Results do not change. */
/* GEMS_OPT_AUTOTUNE (default 1): the first traversal of a 4-state session class (precision,
 * scaling, categories, pattern count to the power of two) with at least 2^22 pattern-updates
 * times every launch shape of the traversal kernel (patterns per lane group x blocks per SM; all
 * give the same values) and keeps the fastest for the process; 0 keeps the default shape (or
 * the one already chosen for the class); 2 + k forces shape k (for comparisons).  No
 * counterpart in the reference.  gems_session_traversal_shape reports the shape in use and
 * whether it was tuned (0 0 0 for the forms that have one shape). */
int gems_session_traversal_shape(gems_session *s, int *patterns_per_group, int *blocks_per_sm,
                                 int *tuned);
int gems_session_set_option(gems_session *s, int option, int value);

/* Tip state bytes [ntaxa][nptn] (PhyloTree::getConvertedSequenceByNumber rows,
 * tree/phylotree.cpp:3331): 0..n-1 states, DNA 4..17 ambiguity bitmask codes, protein
 * 20..22 (B, Z, J), STATE_UNKNOWN (DNA 18, protein 23, else n) for gaps. */
int gems_upload_tips(gems_session *s, const uint8_t *states);
/* ptn_freq[nptn] and ptn_invar[nptn] (phylotreesse.cpp:537,549); invar may be NULL (zeros). */
int gems_upload_patterns(gems_session *s, const double *ptn_freq, const double *ptn_invar);

/* Model: eval[n], evec[n*n], inv_evec[n*n] row-major (ModelSubst getters,
 * model/modelsubst.h:363-371); rates[ncat], props[ncat] (RateHeterogeneity getRate/getProp,
 * model/rateheterogeneity.h:107-172).  Builds the tip tables on the device
 * (phylotreesse.cpp:243-375). */
int gems_set_model(gems_session *s, const double *eval, const double *evec,
                   const double *inv_evec, const double *rates, const double *props);
/* Same, but the FP64 eigendecomposition of the reversible rate matrix runs on the GPU
 * (cyclic Jacobi on the sqrt(pi)-symmetrised matrix; replaces ModelMarkov::decomposeRateMatrix,
 * model/modelmarkov.cpp:1389-1630).  exch_upper holds the n(n-1)/2 exchangeabilities. */
int gems_set_model_from_rates(gems_session *s, const double *exch_upper, const double *freq,
                              const double *rates, const double *props);
/* gems_set_model_from_rates for nsess sessions of one device, state count and category count
 * (at most 128) with every eigendecomposition in one launch, one CTA per model: ModelFinder's
 * candidate models (model/modelfactory.cpp:1263,1367,1558; main/phylotesting.cpp).  Inputs are
 * stacked per session: exch_upper[nsess][n(n-1)/2], freq[nsess][n], rates[nsess][ncat],
 * props[nsess][ncat].  No counterpart in the reference (one decomposition per model). */
int gems_set_model_from_rates_batch(gems_session *const *sessions, int nsess,
                                    const double *exch_upper, const double *freq,
                                    const double *rates, const double *props);
/* New category rates and proportions (rates[ncat], props[ncat]) with the eigensystem kept: what
 * a new Gamma shape or FreeRate parameters change (RateGamma::computeFunction sets the shape,
 * recomputes the rates and clears every partial, model/rategamma.cpp:178-186).  The rates come
 * from the caller, as with gems_set_model.  Partials computed before are stale: clear them in
 * the caller's tree (gems_tree_clear_all_partial_lh) before the next evaluation. */
int gems_set_rates(gems_session *s, const double *rates, const double *props);
/* Copy back the eigensystem in use (for inspection). */
int gems_get_eigensystem(gems_session *s, double *eval, double *evec, double *inv_evec);

/* ---- kernel set ---- */
/* Postorder list of node updates (computePartialLikelihood over all patterns for each
 * entry of traversal_info; tree/phylokernelnew.h:1293-2043). */
int gems_traverse(gems_session *s, const gems_op *ops, int nops);
/* One node update over the patterns [ptn_lower, ptn_upper): the partial of op->dst_slot from
 * its two children, for those patterns only -- PhyloTree::computePartialLikelihood
 * (TraversalInfo &info, size_t ptn_lower, size_t ptn_upper, int packet_id)
 * (tree/phylotree.h:900-903, tree/phylotreesse.cpp:212), which the reference's drivers call
 * once per (packet, traversal entry) (tree/phylokernelnew.h:1274-1281).  Patterns outside the
 * range are left as they are.  ptn_lower must be a multiple of the session's pattern granule,
 * ptn_upper a multiple of it or nptn; the range must be non-empty and inside [0, nptn).
 * Packets that cover [0, nptn) give the same slot contents, bit for bit, as gems_traverse of
 * the same ops. */
int gems_compute_partial(gems_session *s, const gems_op *op, int ptn_lower, int ptn_upper);
/* The pattern granule of gems_compute_partial for this session: 1 for the CUDA-core forms of
 * 4 and 20 states and the generic forms, 128 for the tcgen05 forms (their pattern tiles), the
 * pattern tile of the FP64 61-state GEMM form (the reference's packets are aligned to its
 * vector width in the same way, computeBounds, tree/phylokernelnew.h:1118). */
int gems_session_pattern_granule(gems_session *s, int *granule);
/* Batched traversal over sessions that share one tree (the same op list and lengths) but hold
 * different models -- ModelFinder's candidate models on one alignment (modelfactory.cpp:1558,
 * main/phylotesting.cpp) -- so that many small sessions fill the GPU.  All sessions must have the
 * same device, nptn, nstates, ncat and nslots, at most 128 per call.  61-state mixed SAFE
 * sessions (with tensor cores on) run as one launch over every (session, pattern tile); other
 * forms run one traversal per session.  No counterpart in the reference (it evaluates models
 * one after the other). */
int gems_traverse_batch(gems_session *const *sessions, int nsess, const gems_op *ops, int nops);
/* gems_traverse_batch, then the branch lnL of each session (lnl[nsess]). */
int gems_branch_lnl_batch(gems_session *const *sessions, int nsess, const gems_op *ops, int nops,
                          const gems_branch *br, double *lnl);
/* As gems_branch_lnl_batch with each session's own op list (ops[i], nops[i]) and branch
 * (br[i]): candidates on one tree whose branch lengths differ.  The 61-state mixed form batches
 * when every list has the same length; every session's branch terms are enqueued before any
 * result is read. */
int gems_branch_lnl_batch_ops(gems_session *const *sessions, int nsess, const gems_op *const *ops,
                              const int *nops, const gems_branch *br, double *lnl);
/* Branch log-likelihood (computeLikelihoodBranchSIMD, tree/phylokernelnew.h:2658-3275),
 * after running ops (may be 0).  pattern_lh[nptn] optional (log-likelihood per pattern
 * including the scaling correction). */
int gems_branch_lnl(gems_session *s, const gems_op *ops, int nops, const gems_branch *br,
                    double *lnl, double *pattern_lh);
/* gems_upload_tips + gems_upload_patterns + gems_branch_lnl in one call, with the tip upload
 * overlapped with the traversal: the rows go up in nchunks (1..64) pattern chunks on a second
 * stream and each chunk's traversal starts when its copy is done (4-state sessions, and 20-state
 * sessions with tensor cores off; other forms load first, then evaluate).  Overlap needs pinned
 * host buffers.  A tip byte above STATE_UNKNOWN fails the call with GEMS_ERR_BAD_ARG and leaves
 * the tips invalid, as gems_upload_tips does.  No counterpart in the reference (its alignment is
 * loaded once); replaces reloading the alignment and calling computeLikelihood. */
int gems_branch_lnl_from_host(gems_session *s, const uint8_t *states, const double *ptn_freq,
                              const double *ptn_invar, const gems_op *ops, int nops,
                              const gems_branch *br, int nchunks, double *lnl,
                              double *pattern_lh);
/* Derivatives of lnL w.r.t. the branch length (computeLikelihoodDervSIMD,
 * tree/phylokernelnew.h:2238-2650).  When compute_theta != 0 the ops run first and theta is
 * rebuilt from the two partials (computeLikelihoodBufferSIMD, :2053-2235); otherwise the
 * resident theta is reused at br->length.  df_frac[nptn] (G_matrix row) optional. */
int gems_branch_derv(gems_session *s, const gems_op *ops, int nops, const gems_branch *br,
                     int compute_theta, double *df, double *ddf, double *df_frac);
/* lnL from the resident theta at a new length (computeLikelihoodFromBufferSIMD,
 * tree/phylokernelnew.h:3285-3495). */
int gems_lnl_from_buffer(gems_session *s, double length, double *lnl, double *pattern_lh);
/* Safeguarded Newton on -lnL(t) in [min_len, max_len], starting from guess, over the resident
 * theta of br (rebuilt first when compute_theta != 0).  Same iterate sequence as
 * Optimization::minimizeNewton (utils/optimization.cpp:422-499); the loop runs on the device.
 * opt_len receives the returned length, nevals the number of derivative evaluations. */
int gems_newton_branch(gems_session *s, const gems_op *ops, int nops, const gems_branch *br,
                       int compute_theta, double min_len, double max_len, double xacc,
                       int max_steps, double *opt_len, int *nevals);
/* gems_newton_branch in two halves, so that the Newton loops of many sessions (ModelFinder's
 * candidate models on one tree) run on their streams at the same time: _async enqueues the
 * traversal, theta and the device Newton loop and returns; _wait waits for the session's stream
 * and returns opt_len, nevals and the loop's status.  No counterpart in the reference (it
 * optimises candidates one after the other). */
int gems_newton_branch_async(gems_session *s, const gems_op *ops, int nops,
                             const gems_branch *br, int compute_theta, double min_len,
                             double max_len, double xacc, int max_steps);
int gems_newton_branch_wait(gems_session *s, double *opt_len, int *nevals);

/* ---- allocation-free evaluation ---- */
/* No counterpart in the reference.  lnL at branch length `length` from a theta buffer the
 * caller owns, for callers that cannot allocate device memory when they evaluate: a host whose
 * own memory pool has reserved the device, an embedding that accounts every device byte itself,
 * or a loop that must not hit cudaMalloc/cudaFree (they synchronise the device).  It computes
 * what gems_lnl_from_buffer computes, over caller-owned device arrays:
 * theta[nptn][ncat][nstates] and scale_all[nptn] (the layout gems_get_theta returns),
 * freq[nptn] and invar[nptn] (invar may be NULL); eval[nstates], rates[ncat], props[ncat]
 * are host arrays.  stream is a cudaStream_t (NULL: the default stream).  The call is
 * synchronous: it waits for its stream and writes the result to lnl (host).  No cudaMalloc,
 * cudaFree or allocating library call is made: the reduction scratch is a fixed device array
 * of this library (256 KiB per GPU, held until exit), which limits nptn to 4194304 / G
 * (G = smallest power of two >= ncat); larger calls return GEMS_ERR_BAD_ARG.  The first call
 * on a device looks up the array's device address, so make it before any stream capture on
 * that device.  All calls share the array: calls that overlap on the GPU race and must be
 * serialised by the caller. */
int gems_lnl_from_theta_noalloc(const double *theta, const double *scale_all,
                                const double *freq, const double *invar, int nptn,
                                int nstates, int ncat, const double *eval,
                                const double *rates, const double *props, double length,
                                void *stream, double *lnl);

/* ---- bootstrap reweighting (UFBoot RELL) ---- */
/* Upload R replicates of pattern counts, weights[R][nptn] (FP32), resident until replaced. */
int gems_upload_reweightings(gems_session *s, const float *weights, int R);
/* lnl[r] = sum_p weights[r][p] * pattern_lh[p] for the per-pattern log-likelihoods of the last
 * branch lnL / lnL-from-buffer call: the dotProduct(pattern_lh, boot_sample) of UFBoot
 * (tree/iqtree.cpp:3870-3916, tree/phylokernel.h:65; pattern_lh taken in FP32 as there,
 * accumulated in FP64).  One launch for all R replicates. */
int gems_reweighted_lnl(gems_session *s, double *lnl);
/* Reweighted derivatives of the last gems_branch_derv call: df[r] = sum_p w_rp df_frac_p,
 * ddf[r] = sum_p w_rp (ddf_frac_p - df_frac_p^2). */
int gems_reweighted_derv(gems_session *s, double *df, double *ddf);

/* ---- inspection ---- */
/* partial[nptn * ncat * nstates] (pattern-major, category-major, state-contiguous; FP64
 * values, converted from the session precision) and scale[nptn] (NORM) or [nptn*ncat]
 * (SAFE) counters of a slot.  Either pointer may be NULL. */
int gems_get_partial(gems_session *s, int slot, double *partial, uint16_t *scale);
/* theta[nptn * block] and per-pattern log scale (buffer_scale_all). */
int gems_get_theta(gems_session *s, double *theta, double *scale_all);
/* number of kernel launches issued by this session so far */
int gems_launch_count(gems_session *s, long long *count);
/* Kernel timing with CUDA events on the session stream: when enabled, every launch of the
 * traversal kernel (kernel id 0), branch kernel (1), theta (2), derivative (3),
 * from-buffer (4) and Newton (5) kernels is bracketed by events; gems_profile_read returns the
 * summed device time in ms and the number of timed launches, then resets the counters. */
int gems_profile_enable(gems_session *s, int on);
int gems_profile_read(gems_session *s, int kernel_id, double *total_ms, long long *launches);
/* Alignment ingest on the device: state encoding and pattern compression in the reference's
 * first-appearance order (Alignment::buildPattern / addPatternLazy, alignment.cpp:1240-1268 and
 * :1511-1543; convertState :1856-1958; computeConst :1321-1420).  seqs: host [ntaxa][nsites]
 * characters (encoded = 0; DNA or protein letters as the reference reads them, either case) or
 * state codes (encoded = 1; any state count).  Outputs (host, caller-sized for npat <= nsites):
 * patterns [ntaxa][npat] (row stride npat), weights[npat] (site counts), site_pattern[nsites]
 * and const_char[npat] (may be NULL).  An unrecognised character returns GEMS_ERR_BAD_ARG and
 * names its sequence and site. */
int gems_compress_alignment(int device, int ntaxa, long long nsites, int nstates,
                            const uint8_t *seqs, int encoded, uint8_t *patterns, double *weights,
                            int *site_pattern, uint8_t *const_char, long long *npat);
/* The same ingest kept on the device: gems_ingest_create encodes and compresses (the
 * sequences cross to the GPU once), gems_ingest_read copies any of the results back (NULL to
 * skip), gems_ingest_to_session loads the patterns into a session created with nptn = npat
 * (tips copied on the device and checked as gems_upload_tips does, weights, and ptn_invar from
 * the constant states: computePtnInvar, tree/phylotreesse.cpp:549-612, with p_invar and the
 * model's state frequencies; p_invar = 0 for no +I). */
typedef struct gems_ingest gems_ingest;
int gems_ingest_create(int device, int ntaxa, long long nsites, int nstates, const uint8_t *seqs,
                       int encoded, gems_ingest **out, long long *npat);
int gems_ingest_read(gems_ingest *g, uint8_t *patterns, double *weights, int *site_pattern,
                     uint8_t *const_char);
int gems_ingest_to_session(gems_ingest *g, gems_session *s, double p_invar,
                           const double *state_freq);
void gems_ingest_destroy(gems_ingest *g);
/* Measured compute peaks of a device (no counterpart in the reference: the denominators of the
 * compute rooflines): FP64 and FP32 FMA throughput of the CUDA cores and the dense TF32 rate of
 * the tcgen05 tensor cores, in TFLOP/s.  Takes a few tens of milliseconds. */
int gems_measure_peaks(int device, double *fp64_tflops, double *fp32_tflops, double *tf32_tflops);
/* Runs the time-out path of the bounded grid barrier that the device Newton loop uses (no
 * counterpart in the reference): a two-block cooperative launch waits for a third block that
 * never comes, gives up after about a second and reports GEMS_ERR_TIMEOUT in *status; the
 * device stays usable.  Allocates a few bytes.  For failure-handling tests. */
int gems_check_barrier_timeout(int device, int *status);

/* ---- tree mirror (PhyloTree calls on the path) ---- */
typedef struct gems_tree gems_tree;
/* Unrooted binary tree: leaves 0..ntaxa-1, internal nodes ntaxa..nedges; each node's
 * neighbour order follows the edge order.  The session's nslots chooses the memory mode:
 * ntaxa-2 (one partial per internal node, LM_PER_NODE, tree/phylotree.cpp:905-960);
 * 3*(ntaxa-2) (one per directed branch); or fewer than ntaxa-2, down to
 * floor(log2(ntaxa)) + 1 (LM_MEM_SAVE, tree/memslot.cpp:28-229, tree/phylotree.cpp:1026-1040):
 * a directed branch gets a slot when its partial is computed, a full pool gives up the
 * unlocked slot of the smallest subtree (that partial is recomputed when next needed), and
 * children are traversed larger subtree first.  Fewer slots return GEMS_ERR_ADMISSION, as
 * does a traversal that finds every slot locked.  Results are the same in every mode. */
int gems_tree_create(gems_session *s, int nedges, const int *eu, const int *ev,
                     const double *len, gems_tree **out);
int gems_tree_destroy(gems_tree *t);
int gems_tree_set_branch_limits(gems_tree *t, double min_len, double max_len);
int gems_tree_set_length(gems_tree *t, int u, int v, double len);
int gems_tree_get_lengths(gems_tree *t, double *len); /* in edge order */
int gems_tree_clear_all_partial_lh(gems_tree *t);
/* PhyloTree::computeLikelihood (tree/phylotree.cpp:1258) */
int gems_tree_compute_likelihood(gems_tree *t, double *lnl, double *pattern_lh);
/* computeLikelihoodBranch(dad->findNeighbor(node), dad) */
/* computeLikelihood on new tips, weights and +I terms (every partial recomputed), through
 * gems_branch_lnl_from_host. */
int gems_tree_compute_likelihood_from_host(gems_tree *t, const uint8_t *states,
                                           const double *ptn_freq, const double *ptn_invar,
                                           int nchunks, double *lnl, double *pattern_lh);
int gems_tree_compute_likelihood_branch(gems_tree *t, int node, int dad, double *lnl,
                                        double *pattern_lh);
/* computeLikelihoodDerv(dad->findNeighbor(node), dad) */
int gems_tree_compute_likelihood_derv(gems_tree *t, int node, int dad, double *df, double *ddf);
int gems_tree_compute_likelihood_from_buffer(gems_tree *t, double *lnl);
/* optimizeOneBranch(node1, node2, clearLH, maxNRStep) (tree/phylotree.cpp:2620) */
int gems_tree_optimize_one_branch(gems_tree *t, int node1, int node2, int clear_lh,
                                  int max_nr_step);
/* optimizeAllBranches(my_iterations, tolerance, maxNRStep) (tree/phylotree.cpp:2724) */
int gems_tree_optimize_all_branches(gems_tree *t, int iterations, double tolerance,
                                    int max_nr_step, double *lnl);
/* optimizeAllBranches on ntrees trees of one topology (built from the same edge list, each on
 * its own session: ModelFinder's candidate models on one tree, model/modelfactory.cpp:1263,1367
 * and main/phylotesting.cpp), lnl[ntrees].  Each tree runs exactly the sequence of
 * gems_tree_optimize_all_branches and ends with the same lengths and lnL; the trees move
 * through the common branch order together and every tree's Newton loop on a branch is
 * enqueued before any result is read, so their device work overlaps.  No counterpart in the
 * reference (it optimises one candidate after the other). */
int gems_tree_optimize_all_branches_batch(gems_tree *const *trees, int ntrees, int iterations,
                                          double tolerance, int max_nr_step, double *lnl);
/* PhyloTree::doNNI (tree/phylotree.cpp:4059-4125): swap subtree a (a neighbour of u) with
 * subtree b (a neighbour of v) across the internal branch (u, v); partials and lengths move
 * with their subtrees, the partials looking back across u or v are invalidated.  The edge
 * list reported by gems_tree_get_edges changes accordingly. */
int gems_tree_nni(gems_tree *t, int u, int v, int a, int b);
/* PhyloTree::computeLikelihood of ntrees trees (one per session, sessions as required by
 * gems_branch_lnl_batch_ops) evaluated together: each tree's stale partials and its branch,
 * then one batched evaluation (lnl[ntrees]).  With gems_set_rates and
 * gems_tree_clear_all_partial_lh it re-evaluates every ModelFinder candidate at a new Gamma
 * shape at once (RateGamma::computeFunction, model/rategamma.cpp:178-186, once per candidate in
 * the reference). */
int gems_tree_compute_likelihood_batch(gems_tree *const *trees, int ntrees, double *lnl);
/* PhyloTree::getBestNNIForBran's evaluation (tree/phylotree.cpp:4176-4420, NNI-5, one
 * evaluation round) on the internal branch (u, v), leaving the tree unchanged: the two NNIs --
 * u's neighbour a (the smaller of u's other two) swapped with each of v's other neighbours b,
 * in id order -- each swapped in, its five branches optimised by Newton (max_nr_step steps;
 * the reference's NNI_MAX_NR_STEP is 10) in the order u's outer two, the central one, v's
 * outer two (outer ones in id order; the reference uses its neighbour order), the partial
 * looking back across each branch cleared before it is optimised, the lnL read from the
 * buffers, and swapped back.  As in the reference the optimised lengths carry over from the
 * first move to the second.  Out: moves[2][2] = (a, b), lnl[2], lens[2][5] = central, u's
 * outer, v's outer.  Apply the better one with gems_tree_nni and gems_tree_set_length.  With
 * one slot per internal node and two spare slots (nslots = internal nodes + 2) the evaluation
 * computes in the spares and every partial of the tree stays valid; otherwise the partials
 * whose slots it used are recomputed when next needed. */
int gems_tree_nni_evaluate(gems_tree *t, int u, int v, int max_nr_step, int *moves, double *lnl,
                           double *lens);
/* The SPR move of PhyloTree::assessSPRMove (tree/phylotree.cpp:4822-4880): the subtree at node
 * is pruned from the internal node dad, whose two other neighbours s1 < s2 (by node id) are
 * joined by one branch of their summed length, and dad is inserted into the branch
 * (node2, dad2) -- which must lie outside the pruned subtree and not touch dad -- with half the
 * branch's length on each side.  Edges reported by gems_tree_get_edges: (dad, s1) becomes
 * (s1, s2), (dad, s2) becomes (dad, dad2), (node2, dad2) becomes (dad, node2).  Partials whose
 * subtree is unchanged stay valid; every partial whose subtree holds dad before or after the
 * move is recomputed by the next evaluation.  The reference's SPR search (swapSPR) applies the
 * same move and then optimises the branches (node, dad), (dad2, dad), (node2, dad), (s1, s2)
 * with optimizeOneBranch (tree/phylotree.cpp:4764-4768).  GEMS_ERR_BAD_ARG for a move that
 * does not satisfy the conditions (the tree is unchanged). */
int gems_tree_spr(gems_tree *t, int node, int dad, int node2, int dad2);
/* current edge list (same order as at creation; endpoints change with NNI and SPR moves) */
int gems_tree_get_edges(gems_tree *t, int *eu, int *ev);
/* PhyloTree::computeFuncDerv (tree/phylotree.cpp:2555): set the length of branch
 * (node1, node2) to value without invalidating partials and return f = -dlnL/dt,
 * df = -d2lnL/dt2; new_branch != 0 rebuilds theta for this branch first.  Used to drive a
 * Newton iteration from outside, e.g. in lock-step over pattern shards. */
int gems_tree_compute_func_derv(gems_tree *t, int node1, int node2, double value,
                                int new_branch, double *f, double *df);
/* partial of directed branch dad->node (subtree at node), if valid */
int gems_tree_get_partial(gems_tree *t, int node, int dad, double *partial, uint16_t *scale);
/* partial recomputations (traversal ops) executed so far, and Newton evaluations of the
 * last optimize_one_branch */
int gems_tree_stats(gems_tree *t, long long *partial_ops, int *last_newton_evals);

#ifdef __cplusplus
}
#endif
#endif
