/* exafmm_b200.h -- C ABI of the B200 Laplace FMM engine.
 *
 * One opaque context per caller thread owns a CUDA stream and every device
 * buffer of a solve.  Calls on one context are ordered; a context must not be
 * used from two threads at once (the reference's Kernel/Traversal objects are
 * not re-entrant either).  Every entry point returns 0 on success and a
 * non-zero status otherwise, with the text available from
 * exafmm_last_error().  No C++ exception crosses this boundary.  There is no
 * CPU fallback: without a usable CUDA device, exafmm_create() fails.
 *
 * Data conventions
 *   bodies   xyzq[4*i + {0,1,2,3}] = x, y, z, charge, caller order
 *   results  trg[4*i + {0,1,2,3}]  = potential, d/dx, d/dy, d/dz (the gradient
 *            of the potential, which is what the reference stores in
 *            Body::TRG[1..3]), caller order
 *   bounds   {Xmin[3], Xmax[3]}
 *   cells    ints C x 5 = IPARENT, ICHILD, NCHILD, IBODY, NBODY;
 *            reals C x 4 = X, Y, Z, R   (reference Cell layout, cell 0 = root)
 *   expansions interleaved (re, im), C x NTERM, NTERM = P(P+1)/2,
 *            coefficient (n, m >= 0) at n(n+1)/2 + m
 *
 * Each declaration names the reference interface it stands in for
 * (paths inside the exafmm-beta tree).
 */
#ifndef EXAFMM_B200_H
#define EXAFMM_B200_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct exafmm_ctx exafmm_ctx;

enum {
  EXAFMM_FP64 = 0,  /* plain method: every operator in FP64 */
  EXAFMM_MIXED = 1  /* P2P and M2L in FP32 with compensated accumulation; FP64 at the root levels */
};

/* Kernel(P, eps2, wavek) + Traversal(kernel, theta, nspawn, images, path)
 * + BuildTree(ncrit) (kernels/laplace.h:116, include/traversal.h:291,
 * include/build_tree.h:183).  cycle is the periodic box edge (examples/fmm.cxx:14).
 * device < 0 selects the current device. */
int exafmm_create(exafmm_ctx **ctx, int P, double theta, int ncrit, int nspawn, int images, double cycle,
                  int precision, int device);
int exafmm_destroy(exafmm_ctx *ctx);
const char *exafmm_last_error(const exafmm_ctx *ctx);
/* Error text of the last failed exafmm_create on this thread. */
const char *exafmm_create_error(void);

/* Change the solve parameters of an existing context (the arguments of
 * Kernel/Traversal/BuildTree, as in exafmm_create).  Takes effect at the next
 * build/upward/traverse call; results of earlier steps that depend on a
 * changed parameter must be recomputed. */
int exafmm_set_params(exafmm_ctx *ctx, int P, double theta, int ncrit, int nspawn, int images, double cycle);

/* Mixed form only: which operators run in FP32 and which M2L pairs may
 * (target level >= min_level, |level difference| <= max_dl); the rest runs in
 * FP64.  m2l_fp32: 0 = FP64; 1 = FP32, with the pairs of frequent offset
 * classes evaluated as dense per-class products on the tensor cores (three
 * bf16 pieces per operand, FP32 accumulation) when the system is large
 * enough for that to pay (P = 8 or 10) or periodic (images > 0, any size and
 * P = 4, 6, 8, 10, for accuracy); 2 = FP32 pair by pair only; 3 = as 1
 * with the per-class products at any size; 4 and 5 = as 1 and 3 with the
 * per-class products in FP32 on the CUDA cores.  p2p_fp32: 0 or 1.
 * Defaults: 1, 1, 2, 3 (levels 0 and 1, the root levels, stay FP64).  No
 * counterpart in the reference (its precision is a compile-time switch,
 * EXAFMM_SINGLE). */
int exafmm_set_mixed_policy(exafmm_ctx *ctx, int m2l_fp32, int p2p_fp32, int min_level, int max_dl);
/* Mixed form: how many targets each lane of the FP32 P2P holds (the lanes of
 * a warp split into groups of 4, 8, 16 or 32 by leaf size; each lane takes
 * tpl targets of its group's slice): 0 (default) chooses 2 or 3 per leaf by
 * which fills the slots better, 2 or 3 use that for every leaf.  A tuning
 * parameter (the batch autotuner tries it); results stay within the precision
 * bar either way, though their bits differ.  No counterpart in the reference
 * (its P2P is a SIMD loop over targets, kernels/laplace.h:150-235). */
int exafmm_set_p2p_targets_per_lane(exafmm_ctx *ctx, int tpl);

/* Separate source bodies (examples/fmm.cxx -j IneJ, :37-47, :61-73): the next
 * solves evaluate the field of these n sources (n x 4: x, y, z, q, caller
 * order) at the context's bodies.  As there, the bounds are the targets'
 * extended by the sources (BoundBox::getBounds(jbodies, bounds)), each set gets
 * a tree on those bounds and its upward pass, and the traversal runs target
 * cells against source cells.  Free space; FP64, or the mixed form (FP32 P2P
 * and pair-by-pair FP32 M2L across the two trees, FP64 at the root levels).
 * xyzq == NULL returns to sources == targets. */
int exafmm_set_sources(exafmm_ctx *ctx, const double *xyzq, long long n);
/* The source tree of the last build: cell count, cell table (as
 * exafmm_get_cells) and the sources' tree-order permutation; any output may be NULL. */
int exafmm_get_source_cells(exafmm_ctx *ctx, long long *ncells, int *ints, double *reals, int *perm);

/* Bodies in caller order (Dataset::initBodies / Bodies, include/types.h:72-86).
 * The _device form takes a device pointer to n x 4 doubles on the context's device. */
int exafmm_set_bodies(exafmm_ctx *ctx, const double *xyzq, long long n);
int exafmm_set_bodies_device(exafmm_ctx *ctx, const double *d_xyzq, long long n);

/* A forest of independent systems solved together (no counterpart in the
 * reference, which solves one system per process, examples/fmm.cxx:163-179).
 * count systems, system s holding n[s] bodies; xyzq holds them concatenated in
 * system order (sum n[s] x 4 doubles, caller order inside each system).  The
 * next build / solve gives every system its own bounds (BoundBox::getBounds),
 * tree (BuildTree::buildTree), lists (Traversal::traverse from its own root
 * pair) and expansions, exactly as a solo solve of that system gives them, but
 * every phase runs once for all systems: one set of launches and host read
 * backs per forest, not per system.  Results (exafmm_get_results) are
 * concatenated the same way.  Cells of system s are [cell_base[s],
 * cell_base[s+1]) of the context's cell table, in the layout of its solo tree
 * shifted by cell_base[s]; IBODY and the permutation are offsets into the
 * concatenated bodies.  Free space only (images = 0), sources == targets;
 * empty systems are allowed.  exafmm_set_bodies returns to one system.  The
 * _device form takes the concatenated bodies as a device pointer. */
int exafmm_set_systems(exafmm_ctx *ctx, int count, const long long *n, const double *xyzq);
int exafmm_set_systems_device(exafmm_ctx *ctx, int count, const long long *n, const double *d_xyzq);
/* Layout of a forest after its build: cell_base (count + 1), body_off
 * (count + 1) and each system's bounds (count x 6, as exafmm_get_bounds);
 * any output may be NULL (body_off is known before a build). */
int exafmm_get_systems(exafmm_ctx *ctx, long long *cell_base, long long *body_off, double *bounds);
/* The same forest with one pointer per system instead of the concatenation:
 * xyzq[s] holds system s's n[s] x 4 doubles, trg[s] receives its n[s] x 4
 * results, in host or device memory (each copied with cudaMemcpyDefault, so
 * host pointers must be addressable by CUDA: any pageable or pinned memory).
 * A NULL pointer is allowed only for an empty system.  No counterpart in the
 * reference (one system per process, examples/fmm.cxx:163-179). */
int exafmm_set_systems_list(exafmm_ctx *ctx, int count, const long long *n, const double *const *xyzq);
int exafmm_get_results_list(exafmm_ctx *ctx, double *const *trg);

/* Repeated MD-style solves without a host round trip (no counterpart in the
 * reference, whose MD wrappers re-partition and re-upload every step,
 * wrappers/gromacs.cxx:139-190): every body's position moves in place on the
 * device by sigma times three standard normals drawn from a counter-based
 * stream (SplitMix64 words by (seed, body index), Box-Muller), so the move
 * depends only on (seed, sigma, body index); the next solve rebuilds the tree
 * on the device.  An MD code that integrates on the GPU passes its new
 * positions with exafmm_set_bodies_device instead. */
int exafmm_displace_bodies(exafmm_ctx *ctx, double sigma, unsigned long long seed);
/* The context's current bodies (caller order, n x 4), to host or device memory. */
int exafmm_get_bodies(exafmm_ctx *ctx, double *xyzq);
int exafmm_get_bodies_device(exafmm_ctx *ctx, double *d_xyzq);

/* BoundBox::getBounds(Bodies&) (include/bound_box.h:11-25), including its
 * sequential 1e-5 drift, evaluated on the device in closed form; with separate
 * sources, extended by them as getBounds(jbodies, bounds) does
 * (bound_box.h:28-36), which is what the solve uses. */
int exafmm_get_bounds(exafmm_ctx *ctx, double *bounds6);

/* BuildTree::buildTree(bodies, buffer, bounds) (include/build_tree.h:186-209).
 * bounds6 == NULL computes them as examples/fmm.cxx:163 does. */
int exafmm_build_tree(exafmm_ctx *ctx, const double *bounds6);

/* UpDownPass::upwardPass (include/up_down_pass.h:49-60). */
int exafmm_upward(exafmm_ctx *ctx);

/* Traversal::traverse(cells, cells, cycle, dual) (include/traversal.h:326-352):
 * builds the M2L/P2P lists and evaluates them; clears the results first, as
 * Dataset::initTarget does before a solve.  With images > 0 the lists cover the
 * 27 nearest images of the root, and images > 1 adds the lattice of
 * Traversal::traversePeriodic (include/traversal.h:233-287) in FP64. */
int exafmm_traverse(exafmm_ctx *ctx);

/* UpDownPass::downwardPass (include/up_down_pass.h:63-75). */
int exafmm_downward(exafmm_ctx *ctx);

/* Bounds + build + upward + traverse + downward, the examples/fmm.cxx:163-179 loop body. */
int exafmm_solve(exafmm_ctx *ctx);

/* UpDownPass::getDipole(bodies, X0) (include/up_down_pass.h:78-86): sum of
 * (x_i - X0) q_i over the context's bodies, FP64 on the device.  X0 == NULL is
 * the origin. */
int exafmm_get_dipole(exafmm_ctx *ctx, const double *X0, double *dipole3);
/* UpDownPass::dipoleCorrection(bodies, dipole, numBodies, cycle)
 * (include/up_down_pass.h:89-99) applied to the results of the last solve:
 * pot -= 4 pi / (3 cycle^3) |dipole|^2 / numBodies / q_i, grad -= 4 pi / (3 cycle^3) dipole.
 * As in the reference, a zero charge makes its potential non-finite. */
int exafmm_dipole_correction(exafmm_ctx *ctx, const double *dipole3, long long num_bodies);

/* Results (Body::TRG scattered back by IBODY).  The _device form writes n x 4
 * doubles to a device pointer. */
int exafmm_get_results(exafmm_ctx *ctx, double *trg);
int exafmm_get_results_device(exafmm_ctx *ctx, double *d_trg);

/* Tree and list inspection for parity checks. */
int exafmm_tree_info(exafmm_ctx *ctx, long long *ncells, int *depth, long long *n_m2l, long long *n_p2p);
/* Pair interactions of the last solve's P2P lists: the sum over list entries
 * (target cell i, source cell j) of NBODY(i) * NBODY(j), self pairs included
 * (the work the P2P kernels do; kernels/laplace.h:150-235 per call).  Counted
 * on the device from the lists.  No counterpart in the reference (its
 * EXAFMM_COUNT_KERNEL build counts calls, include/traversal.h:396-410). */
int exafmm_list_work(exafmm_ctx *ctx, long long *p2p_interactions);
int exafmm_get_cells(exafmm_ctx *ctx, int *ints, double *reals);
/* perm[i] = caller index of the body in tree slot i (Body::IBODY after buildTree). */
int exafmm_get_perm(exafmm_ctx *ctx, int *perm);
/* Pairs (target cell, source cell, periodic image 0..26, 13 = unshifted), grouped by target. */
int exafmm_get_lists(exafmm_ctx *ctx, int *m2l, int *p2p);
int exafmm_get_expansions(exafmm_ctx *ctx, double *M, double *L);

/* The CUDA stream (cudaStream_t) the context runs on. */
void *exafmm_stream(exafmm_ctx *ctx);
/* Device time (ms, CUDA events on the context's stream) of the phases of the
 * last solve: bounds, tree, upward, lists, m2l, p2p, downward, total. */
int exafmm_phase_times(exafmm_ctx *ctx, double *ms8);
/* Solve records in the reference's file formats.  exafmm_write_list writes
 * path + "list%06d.dat" (rank) as Traversal::writeList does under
 * EXAFMM_COUNT_LIST (include/traversal.h:412-421): per cell, in cell order, the
 * Morton key ICELL (BuildTree::getKey, include/build_tree.h:111-120), the P2P
 * and the M2L list sizes of the last traversal.  exafmm_write_time writes
 * path + "time%06d.dat" as logger::writeTime does (include/logger.h:116-127):
 * the solve phases timed since the last call, summed, in seconds, under the
 * reference's event names (Get bounds, Grow tree, Link tree, Upward pass,
 * Traverse, Traverse periodic when periodic, Downward pass), then clears them.
 * exafmm_write_time_events writes given events in that format (events with the
 * same name add up, as logger::stopTimer accumulates).  path is a directory
 * prefix ending in '/' ("./" if null). */
int exafmm_write_list(exafmm_ctx *ctx, const char *path, int rank);
int exafmm_write_time(exafmm_ctx *ctx, const char *path, int rank);
/* The same events handed to the caller instead of a file (what the reference's
 * logger::timer holds after these calls, include/logger.h:39-53): *count is
 * the number of events; with names (cap x 32 chars, NUL-terminated) and
 * seconds given, cap >= *count, they are filled in the name order and the
 * engine's timers are cleared.  Waits for the phases timed so far. */
int exafmm_take_timers(exafmm_ctx *ctx, int cap, char *names, double *seconds, int *count);
int exafmm_write_time_events(const char *path, int rank, int count, const char *const *names, const double *seconds);
/* BuildTree::getKey (include/build_tree.h:111-120) of center X at level, cube
 * corner Xmin and cell diameter, with the compiled reference's 32-bit shift
 * semantics (keys of levels >= 11 wrap as they do there). */
unsigned long long exafmm_morton_key(const double *X, const double *Xmin, double diameter, int level);

/* Device memory held by the context's grow-only buffers, in bytes (no
 * counterpart in the reference; used by the request server's admission). */
int exafmm_device_bytes(exafmm_ctx *ctx, long long *bytes);
/* Kernels this library has launched in this process (all contexts). */
long long exafmm_launch_count(void);

/* Traversal::direct (include/traversal.h:355-377): FP64 direct sum of all
 * sources onto the targets over the periodic image range of images/theta.
 * Host arrays; trg accumulates. */
int exafmm_direct(const double *targets, long long nt, const double *sources, long long ns, int images,
                  double theta, double cycle, double *trg);
/* The same sum over the images -prange..prange in each direction (the range
 * the MD wrappers' direct sums use, wrappers/gromacs.cxx:289-301: prange =
 * sum of 3^i over the image levels). */
int exafmm_direct_range(const double *targets, long long nt, const double *sources, long long ns, int prange,
                        double cycle, double *trg);
/* The cutoff direct sum of wrappers/md_distributed.cxx:407-461 (FMM_Cutoff):
 * pairs at images -prange..prange per direction (shifts i * cycle3[d] rounded
 * to float, as there) closer than cutoff; FP64 on the device.  Host arrays;
 * trg accumulates (potential, gradient). */
int exafmm_direct_cutoff(const double *targets, long long nt, const double *sources, long long ns, int prange,
                         const double *cycle3, double cutoff, double *trg);

/* Ewald summation (include/ewald.h:7-197, as examples/ewald.cxx drives it), FP64
 * on the device: wave part over the integer waves |k| <= ksize of
 * Ewald::initWaves, real part (erfc) over pairs closer than cutoff at their
 * nearest periodic image, self term.  alpha and sigma as in Ewald's
 * constructor; cycle = box edge, bodies taken modulo the box.  Host arrays;
 * trg accumulates (potential, gradient) in caller order. */
int exafmm_ewald(const double *xyzq, long long n, int ksize, double alpha, double sigma, double cutoff, double cycle,
                 double *trg);
const char *exafmm_ewald_error(void);

/* Error text of the last failed exafmm_direct / exafmm_kernel_* call on this thread. */
const char *exafmm_kernel_error(void);

/* Per-operator forms (the examples/kernel.cxx known-answer chain,
 * kernels/laplace.h:150-388).  Host arrays; outputs accumulate. */
int exafmm_kernel_p2m(int P, const double *X, long long n, const double *xyzq, double *M);
int exafmm_kernel_m2m(int P, const double *Xp, int nchild, const double *Xc, const double *Mc, double *Mp);
int exafmm_kernel_m2l(int P, const double *Xi, const double *Xj, const double *Mj, double *Li,
                      const double *Xperiodic);
int exafmm_kernel_l2l(int P, const double *Xc, const double *Xp, const double *Lp, double *Lc);
int exafmm_kernel_l2p(int P, const double *X, const double *L, long long n, const double *xyzq, double *trg);
int exafmm_kernel_p2p(long long ni, const double *xi, long long nj, const double *xj, const double *Xperiodic,
                      double *trg);

/* ---- Batched and served solves (no counterpart in the reference, which
 * solves one system per process, examples/fmm.cxx:163-179) ----
 *
 * Both run a pool of `workers` solve contexts, each on its own host thread and
 * CUDA stream, so independent systems overlap on the GPU.  A system's results
 * do not depend on what else runs: every reduction of a solve has a fixed
 * order, so its bits are the same alone, in a batch or beside other requests. */
typedef struct exafmm_batch exafmm_batch;
int exafmm_batch_create(exafmm_batch **b, int P, double theta, int ncrit, int nspawn, int precision, int device,
                        int workers);
int exafmm_batch_destroy(exafmm_batch *b);
const char *exafmm_batch_error(const exafmm_batch *b);
/* Solves count systems (n[i] bodies at xyzq[i], results to trg[i], caller
 * order, host memory); blocks until all are done.  Largest systems first. */
int exafmm_batch_solve(exafmm_batch *b, int count, const long long *n, const double *const *xyzq,
                       double *const *trg);
/* Device time (ms) of each system of the last exafmm_batch_solve. */
int exafmm_batch_times(exafmm_batch *b, double *ms);
/* enable != 0: the following solves try ncrit 32, 64 and 128 on the first
 * systems of each size class (floor(log2 n)) and keep the fastest per body;
 * enable == 0 freezes the table found so far (systems of classes without an
 * entry use the batch's ncrit). */
int exafmm_batch_autotune(exafmm_batch *b, int enable);
/* The tuned table as (size class, ncrit) pairs; returns the number of pairs. */
int exafmm_batch_ncrit_table(exafmm_batch *b, int *pairs, int cap);
/* Replaces the table with k (size class, ncrit) pairs and freezes it (so two
 * batches can solve on the same trees). */
int exafmm_batch_set_ncrit_table(exafmm_batch *b, const int *pairs, int k);
/* Forest mode (buckets > 0): the systems of one call are cut into at most
 * `buckets` groups of whole size classes with about equal bodies each
 * (exafmm_forest_buckets), and every group is solved as one forest
 * (exafmm_set_systems_list) on one worker context: every phase launches once
 * per group, not once per system, and the groups run concurrently.  Each
 * system's results are the bits of its solo solve at the group's ncrit.  The
 * autotuner keys a group by the lowest size class it holds and tries one
 * candidate per call.  In forest mode xyzq[i] and trg[i] may be host or device
 * pointers.  buckets == 0 (the default) solves one system per context. */
int exafmm_batch_set_forest(exafmm_batch *b, int buckets);
/* exafmm_set_mixed_policy for every context of the batch (mixed precision). */
int exafmm_batch_set_mixed_policy(exafmm_batch *b, int m2l_fp32, int p2p_fp32, int min_level, int max_dl);
/* The autotuner's ncrit candidates (k of them, tried in this order; default
 * 32, 64, 128); setting them restarts the tuning of every class. */
int exafmm_batch_set_ncrit_candidates(exafmm_batch *b, const int *ncrit, int k);
/* The autotuner's P2P targets-per-lane candidates (exafmm_set_p2p_targets_per_lane:
 * 0, 2, 3; default 0 alone): it tries every ncrit candidate with each of them
 * (one per call), and keeps the fastest pair per class. */
int exafmm_batch_set_p2p_candidates(exafmm_batch *b, const int *tpl, int k);
/* The tuned table as (size class, ncrit, targets per lane) triples; returns
 * the number of classes.  The _set form loads such a table and freezes it. */
int exafmm_batch_config_table(exafmm_batch *b, int *triples, int cap);
int exafmm_batch_set_config_table(exafmm_batch *b, const int *triples, int k);
/* Forest mode: each group's targets per lane in the last call (up to cap);
 * returns the number of groups. */
int exafmm_batch_bucket_p2p(exafmm_batch *b, int *bucket_tpl, int cap);
/* Forest mode: device time (ms) of the last call, from an event every worker
 * stream waits on before its first copy in to the last group's copy out. */
int exafmm_batch_elapsed(exafmm_batch *b, double *ms);
/* Forest mode: the group of each system of the last call (bucket_of[count])
 * and each group's ncrit (up to cap); returns the number of groups. */
int exafmm_batch_buckets(exafmm_batch *b, int *bucket_of, int *bucket_ncrit, int cap);
/* The grouping itself (host only): non-empty systems' size classes
 * floor(log2 n) in increasing order, cut into at most `buckets` runs of whole
 * classes; group b's share of the bodies ends at (b + 1) / buckets of the
 * total, and the next group starts before a class whose bodies would overshoot
 * that mark by more than stopping short of it falls below.  Empty systems join
 * group 0.  Returns the number of groups, -1 on bad input. */
int exafmm_forest_buckets(int count, const long long *n, int buckets, int *bucket_of);

typedef struct exafmm_server exafmm_server;
/* Request server: submitted systems wait in a FIFO queue and start when their
 * estimated device memory fits beside the requests in flight and the idle
 * contexts' buffers within hbm_budget_bytes (a request is always admitted
 * when nothing else is in flight). */
int exafmm_server_create(exafmm_server **s, int device, int workers, double hbm_budget_bytes);
/* Drains the queue, then stops the workers. */
int exafmm_server_destroy(exafmm_server *s);
/* Queues one system; xyzq and trg (host, n x 4 doubles) must stay valid until
 * the request completes.  *ticket identifies it for poll / wait. */
int exafmm_server_submit(exafmm_server *s, const double *xyzq, long long n, double *trg, int P, double theta,
                         int ncrit, int nspawn, int precision, long long *ticket);
int exafmm_server_poll(exafmm_server *s, long long ticket, int *done);
/* Device-resident repeat chains (an MD trajectory: one system solved step
 * after step while its bodies move; no counterpart in the reference, whose MD
 * wrappers rebuild from host data every step, wrappers/gromacs.cxx:139-190).
 * A session owns one context that keeps the chain's bodies, tree and
 * expansions on the device between steps; between steps its device bytes
 * count against the budget as held.  xyzq (host, n x 4) must stay valid until
 * the first step completes. */
int exafmm_server_open_session(exafmm_server *s, const double *xyzq, long long n, int P, double theta, int ncrit,
                               int nspawn, int precision, long long *session);
/* Queues the session's next step (one at a time per session; status 2 while
 * the previous one is in flight).  The first step solves the opened bodies;
 * each later step first moves them on the device, to d_xyzq (device memory,
 * n x 4) when it is not NULL, else by exafmm_displace_bodies(sigma, seed),
 * and rebuilds the tree there.  Results go to trg (host, n x 4); wait / poll
 * take the ticket as for exafmm_server_submit. */
int exafmm_server_submit_step(exafmm_server *s, long long session, double sigma, unsigned long long seed,
                              const double *d_xyzq, double *trg, long long *ticket);
/* The session's current bodies (host, n x 4); the session must be idle. */
int exafmm_server_session_bodies(exafmm_server *s, long long session, double *xyzq);
/* Releases the session's context (status 2 while a step is in flight). */
int exafmm_server_close_session(exafmm_server *s, long long session);
/* Blocks until the request is done and releases its ticket.  times4: queue
 * wait, start to results on the host, submit to results on the host (ms), and
 * the solve's device time (ms).  Returns the request's status. */
int exafmm_server_wait(exafmm_server *s, long long ticket, double *times4);
/* stats6: bytes in flight, bytes held by idle contexts, peak admitted bytes,
 * completed requests, queued requests, budget. */
int exafmm_server_stats(exafmm_server *s, double *stats6);
/* Continuous batching: a worker that takes a request of at most
 * max_request_bodies bodies also takes the queued requests (in queue order)
 * of at most that size with the same parameters, up to max_requests requests
 * and max_group_bodies bodies in all, each admitted against the budget as it
 * joins, and solves them as one forest (exafmm_set_systems_list): every
 * request gets the bits of its solo solve.  Chain steps are never grouped.
 * max_requests = 1 turns grouping off.  Defaults: 64, 262144, 4194304. */
int exafmm_server_set_grouping(exafmm_server *s, int max_requests, long long max_request_bodies,
                               long long max_group_bodies);
/* exafmm_set_mixed_policy for the server's mixed-precision requests (solves,
 * groups and sessions opened afterwards). */
int exafmm_server_set_mixed_policy(exafmm_server *s, int m2l_fp32, int p2p_fp32, int min_level, int max_dl);
/* Requests solved so far inside a group of two or more. */
int exafmm_server_grouped(exafmm_server *s, long long *requests);
/* Error text of the last failed exafmm_server_wait on this thread. */
const char *exafmm_server_error(void);

/* Allocation-free form of exafmm_get_bounds, for callers that may not allocate
 * device memory (a host framework that owns all device memory through its own
 * pool, or a latency-bound loop that cannot pay for cudaMalloc/cudaFree).  No
 * counterpart in the reference.  d_xyzq: n x 4 doubles on the current device;
 * d_bounds6: 6 doubles on the current device, written on `stream` (a
 * cudaStream_t; NULL is the legacy default stream).  Needs no context and
 * allocates nothing: its only scratch is a 128-byte array built into the
 * library, held by every GPU that loads it until the process exits.  The first
 * call in each CUDA context (per device, and again after cudaDeviceReset or
 * under a caller's own context) looks up that array's address, so make it
 * before any stream capture.  All calls share the array, so calls that overlap
 * on the GPU race.  Returns 0, or 2 when n is outside [0, 2^31 - 1], 3 for a
 * null pointer, 4 for a CUDA error raised by this call, 5 when a CUDA error
 * was already pending on the calling thread (it is left pending, and nothing
 * is launched). */
int exafmm_get_bounds_noalloc(const double *d_xyzq, long long n, double *d_bounds6, void *stream);

/* Host-side closed form of the bounds drift: fl(x -/+ 1e-5) applied k times
 * (up != 0 adds).  Runs on the CPU; exposed so its exactness can be checked
 * without a GPU. */
double exafmm_drift(double x, long long k, int up);

#ifdef __cplusplus
}
#endif
#endif
