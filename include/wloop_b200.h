/*
 * wloop_b200.h -- C ABI of the B200 (sm_100a) implementation of the wloop
 * measurement path: HYP smearing, APE / spatial-HYP smearing of the spatial
 * links, temporal and spatial line products and the time-slice resolved
 * Wilson-loop correlation matrices W(sl1,sl2;t,r;x0).
 *
 * All entry points take plain pointers and sizes.  Functions return 0 on
 * success and -1 on failure; wlg_last_error() then describes the failure
 * (CUDA errors name the kernel).  No entry point falls back to the CPU: with
 * no usable GPU every compute call fails.
 *
 * Host field layout ("AoS lexicographic"): link (s,mu) of site
 * s = x3 + N3*(x2 + N2*(x1 + N1*x0)) is the su3_dble at aos + 18*(4*s+mu),
 * i.e. 9 (re,im) pairs c11..c33.  The openQCD layout of udfld()/alloc_lnk()
 * (8 links per odd point, modules/lnk/lnkcom.c:840-859) is accepted through
 * wlg_upload_openqcd() with the caller's ipt[] table.
 *
 * Boundary conditions: bc = 0 open (temporal links at x0=N0-1 are zero, as
 * openQCD's set_bc() leaves them), bc = 3 periodic.
 *
 * Precision: WLG_FP64 keeps links and staples in FP64 (the reference form).
 * WLG_MIXED stores links and computes staples / line products in FP32 and
 * keeps the SU(3) projection and all loop and plaquette sums in FP64.
 */
#ifndef WLOOP_B200_H
#define WLOOP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Raised from the reference's MAX_SM_LEVELS (5, include/wloop.h:13) so that
 * six-level runs fit. */
#define WLG_MAX_SM_LEVELS 8

#define WLG_FP64 0
#define WLG_MIXED 1

#define WLG_OP_APE 0 /* op_smear_t APE, include/wloop.h:17-21 */
#define WLG_OP_HYP 1 /* op_smear_t HYP */

/* Mirrors wloop_parms_t (include/wloop.h:24-36) without the result pointer. */
typedef struct {
  int msl;                     /* number of smearing levels */
  int nss[WLG_MAX_SM_LEVELS];  /* sweeps added per level (incremental, smear.c:109-120) */
  int mwlt;                    /* maximal temporal extent, 1 <= mwlt <= N0/2+1 */
  int mwlr;                    /* maximal spatial extent,  1 <= mwlr <= Nk/2+1 */
  int op_smear;                /* WLG_OP_APE or WLG_OP_HYP */
  double alpha_action[3];      /* HYP parameters for the static action */
  double alpha_ape;            /* APE parameter for the spatial links */
  double alpha_hyp[2];         /* spatial HYP parameters */
  int proj_iter;               /* projection iterations; projection on iff > 0 */
} wlg_wloop_parms;

typedef struct wlg_ctx wlg_ctx;

/* ---- errors and devices ------------------------------------------------ */
const char* wlg_last_error(void);
int wlg_device_count(void);
int wlg_version(void);

/* ---- context: one lattice resident on one GPU ---------------------------
 * Replaces the module-static state of hyp_links.c, ape_links.c, smear.c and
 * wloop.c (all file-static there, e.g. hyp_links.c:68-73, wloop.c:62-67). */
int wlg_create(const int n[4], int bc, int precision, int device, wlg_ctx** out);
int wlg_destroy(wlg_ctx* ctx);
int wlg_sync(wlg_ctx* ctx);
/* Frees smearing and loop scratch (free_hyp, free_ape_links, free_smear,
 * free_wloop); the gauge field stays. */
int wlg_free_scratch(wlg_ctx* ctx);

/* ---- gauge field transfers ---------------------------------------------- */
int wlg_upload_links(wlg_ctx* ctx, const double* aos);
/* Pipelined upload: wlg_prefetch_links starts the host-to-device copy of the
 * next field (same layout as wlg_upload_links) on the context's copy stream
 * and returns at once, so the copy overlaps a measurement in progress;
 * wlg_upload_prefetched makes it the context's gauge field (ordered after
 * the copy on the context's stream).  The host buffer must stay unchanged
 * until the copy is done (pinned memory makes it asynchronous).  One
 * prefetch at a time. */
int wlg_prefetch_links(wlg_ctx* ctx, const double* aos);
int wlg_upload_prefetched(wlg_ctx* ctx);
int wlg_download_links(wlg_ctx* ctx, double* aos);
int wlg_upload_openqcd(wlg_ctx* ctx, const double* ud, const int* ipt);
int wlg_download_openqcd(wlg_ctx* ctx, double* ud, const int* ipt);
/* Synthetic field on the device (same bytes as wlg_generate_links). */
int wlg_generate(wlg_ctx* ctx, uint64_t seed, double eps);
/* Synthetic field on the host into aos (4*V links).  Link (s,mu) is
 * exp(i eps sum_a h_a lambda_a), h_a ~ N(0,1) from Philox4x32-10 keyed by
 * seed, reunitarised; open bc zeroes the temporal links at x0=N0-1. */
int wlg_generate_links(const int n[4], int bc, uint64_t seed, double eps, double* aos);
/* Uniform [0,1) draw used for per-configuration parameters. */
double wlg_aux_uniform(uint64_t seed, uint64_t index, uint32_t tag);

/* ---- smearing ------------------------------------------------------------
 * HYP smearing of the links of directions [mu0,mu1) in place
 * (hyp_links: 0,4; hyp_time_links: 0,1; hyp_space_links: 1,4;
 *  modules/smear/hyp_links.c:398-472).  Skipped when a1 == 0 (:405). */
int wlg_hyp(wlg_ctx* ctx, double a1, double a2, double a3, int proj, int piter, int mu0, int mu1,
            int keep);
/* nsweeps APE sweeps U <- P[U + alpha * staples] (ape_links.c:217-284);
 * time = 1 smears all four directions, time = 0 only the spatial ones. */
int wlg_ape(wlg_ctx* ctx, double alpha, int proj, int piter, int time, int nsweeps, int keep);
/* nsweeps two-level spatial HYP sweeps (hyp_spatial_links.c:289-344). */
int wlg_hyp_spatial(wlg_ctx* ctx, double a1, double a2, int proj, int piter, int nsweeps,
                    int keep);
/* Sum of Re tr U(p) over all plaquettes (lnk_plaq_sum, lnkplaq.c:117-128). */
int wlg_plaq_sum(wlg_ctx* ctx, double* out);

/* ---- Wilson loops ----------------------------------------------------------
 * wloop_sum on the current (HYP-smeared) field: spatial smearing levels
 * (smear.c:99-121), then for r,t all msl x msl loops per time slice
 * (wloop.c:524-608).  wl_mat receives msl*msl*mwlt*mwlr*N0 doubles at
 * wl_idx(sl1,sl2,t,r,x0) = sl1+msl*(sl2+msl*(t+mwlt*(r+mwlr*x0)))
 * (wloop_parms.c:431-434).  plaq (optional, msl doubles) receives the
 * plaquette sum after each level. */
int wlg_wloop_sum(wlg_ctx* ctx, const wlg_wloop_parms* p, double* wl_mat, double* plaq);
/* HYP (alpha_action, all directions, as ms10 set_data does: main/ms10.c:633-646)
 * followed by wlg_wloop_sum. */
int wlg_measure(wlg_ctx* ctx, const wlg_wloop_parms* p, double* wl_mat, double* plaq);
/* Only the smearing levels of wlg_wloop_sum (smear(), smear.c:99-121). */
int wlg_smear_levels(wlg_ctx* ctx, const wlg_wloop_parms* p, double* plaq);
/* Level store after wlg_smear_levels / wlg_wloop_sum: spatial links of
 * level sl in AoS [V][3][18] (get_pus slots 0..msl-1, smear.c:124-127). */
int wlg_download_level(wlg_ctx* ctx, int sl, double* aos3);
/* Spatial lines of level sl left by the last wlg_wloop_sum (length *length
 * = mwlr >= 2; get_pus slots msl..2msl-1 after wloops). */
int wlg_download_lines(wlg_ctx* ctx, int sl, double* aos3, int* length);

/* ---- single-field kernels of the lnk/smear API ------------------------------
 * vb(x,mu) += staples of the (mu,nu) plane, nu-links from u1, mu-links from
 * u2 (staple_sum, staple_sum.c:53-87); fields in AoS lexicographic layout. */
int wlg_staple_sum(const int n[4], const double* u1, const double* u2, int mu, int nu, double* vb);
/* In-place projection of nmat packed su3_dble matrices
 * (approx_project_to_su3_dble, projection.c:120-154). */
int wlg_project(double* mats, int nmat, int iter);
/* v[i] += staple of the link triple (u1[i],u2[i],u3[i]) for nmat packed
 * su3_dble: dn = 0 up staple u1 u2 u3^dag, dn = 1 down staple u1^dag u2 u3;
 * save = 1 general 3x3 form (add_*_staple_lnks_save, lnkstaple.c:385-410),
 * save = 0 SU(3) form with the third column rebuilt (add_*_staple_lnks,
 * lnkstaple.c:296-315). */
int wlg_staples(int nmat, const double* u1, const double* u2, const double* u3, double* v, int dn,
                int save);

/* ---- batches: many configurations measured in one CUDA-graph launch --------
 * No counterpart in the reference (ms10 measures one configuration at a
 * time, main/ms10.c:701-742).  A batch holds nconf configurations of
 * possibly different lattices (dims[4*c..4*c+3], bcs[c], parms[c]) on one
 * GPU; wlg_batch_run applies to every one of them what wlg_measure applies to
 * one (HYP with alpha_action, the smearing levels, all Wilson loops) with each
 * stage as one kernel over all configurations, the whole sequence captured
 * into a CUDA graph on the first run and replayed afterwards. */
typedef struct wlg_batch wlg_batch;
int wlg_batch_create(int nconf, const int* dims, const int* bcs, const wlg_wloop_parms* parms,
                     int precision, int device, wlg_batch** out);
int wlg_batch_destroy(wlg_batch* b);
int wlg_batch_size(wlg_batch* b);
/* device bytes held by the batch's field arena */
long long wlg_batch_bytes(wlg_batch* b);
/* gauge field of configuration i from a host AoS su3_dble buffer */
int wlg_batch_upload(wlg_batch* b, int i, const double* aos);
/* synthetic fields for all configurations on the device */
int wlg_batch_generate(wlg_batch* b, const uint64_t* seeds, const double* eps);
int wlg_batch_snapshot(wlg_batch* b);
int wlg_batch_restore(wlg_batch* b);
/* measure every configuration (synchronous); results via wlg_batch_result */
int wlg_batch_run(wlg_batch* b);
int wlg_batch_result(wlg_batch* b, int i, double* wl_mat);
/* device time of the last run and kernels per run */
int wlg_batch_stats(wlg_batch* b, double* last_ms, int* kernels_per_run);
void* wlg_batch_stream(wlg_batch* b);
/* Device memory of batches comes from a stream-ordered pool per device that
 * keeps what batches free for the next batch; this is how much of it is idle
 * (free for batches, not visible to cudaMemGetInfo). */
long long wlg_batch_pool_idle_bytes(int device);
/* contraction shape for the whole batch (0 = automatic); G <= 4; SB selects
 * the form: 1 or 2 the third (SB levels per reduction), 0 the fourth, 3 the
 * fourth with its level loops unrolled (msl 4-6), 4 the fourth with bulk-copy
 * staging of the top lines (lattices whose time slice is not a whole number
 * of 32-site tiles run the fourth), 5 SB 3 with the FP32 products as packed
 * two-lane FMAs (FP32 batches; an FP64 batch runs SB 3) */
int wlg_batch_set_contract_shape(wlg_batch* b, int G, int SB, int nCB, int block);
/* on (default): the first run executes directly and captures the pipeline,
 * later runs replay the graph; off: every run executes directly */
int wlg_batch_use_graph(wlg_batch* b, int on);
/* device bytes a batch of these configurations would hold, or -1 */
long long wlg_batch_estimate_bytes(int nconf, const int* dims, const int* bcs,
                                   const wlg_wloop_parms* parms, int precision);

/* ---- serving: a request loop with continuous batching -----------------------
 * No counterpart in the reference.  Requests queue FIFO; max_inflight worker
 * threads each take the oldest request whose device footprint fits the
 * budget (mem_fraction of the HBM free at creation, minus batches in flight)
 * and the memory free now, plus later pending requests of the same precision
 * (any lattices; up to max_batch) that fit as well, and measure them as one
 * wlg_batch on their own stream, so batches of different workers overlap on
 * the device and new requests are admitted as soon as a worker and memory
 * free up.  A head of the queue that does not fit yet is bypassed by later
 * requests only until it has waited the bypass limit (wlg_server_set_limits),
 * so it cannot starve. */
typedef struct {
  int n[4];
  int bc;
  wlg_wloop_parms parms;  /* alpha_action: HYP of the gauge field, as wlg_measure */
  int precision;          /* WLG_FP64 or WLG_MIXED */
  uint64_t seed;          /* synthetic field (wlg_generate_links) when links == NULL */
  double eps;
  const double* links;    /* optional host AoS su3_dble field, copied at submission */
} wlg_request;
typedef struct wlg_server wlg_server;
int wlg_server_create(int device, double mem_fraction, int max_inflight, int max_batch,
                      wlg_server** out);
int wlg_server_destroy(wlg_server* s);
/* returns the request id (> 0) or -1 */
long long wlg_server_submit(wlg_server* s, const wlg_request* r);
/* blocks until request id is done; wl_mat (may be NULL) gets its result */
int wlg_server_wait(wlg_server* s, long long id, double* wl_mat, double* latency_ms,
                    int* batch_size);
int wlg_server_release(wlg_server* s, long long id);
const char* wlg_server_error(void);
/* latency percentiles over completed requests (submission to result on the
 * host) and completed requests per second since the first submission */
int wlg_server_stats(wlg_server* s, long long* completed, long long* failed, long long* batches,
                     double* p50_ms, double* p99_ms, double* throughput);
long long wlg_server_budget(wlg_server* s);
/* Replaces the memory budget (budget_bytes > 0) and the bypass limit
 * (bypass_ms >= 0; default 5000): a request at the head of the queue that
 * does not fit yet lets later requests that fit start before it until it has
 * waited bypass_ms, after which nothing else starts before it. */
int wlg_server_set_limits(wlg_server* s, long long budget_bytes, double bypass_ms);

/* ---- plaquette sum without device allocation -------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory at this point (memory owned by another allocator or a preallocated
 * arena; a latency-critical path where cudaMalloc/cudaFree would synchronise
 * the device): the same sum as wlg_plaq_sum, from a su3_dble field the caller
 * already holds in device memory.  links: 4*V links in AoS lexicographic order
 * (device or managed memory); out: one double in device memory, written when
 * the work on `stream` (a cudaStream_t, 0 = default stream) completes.
 * Its only scratch is a fixed array inside the library (128 KiB per GPU that
 * loads the library, held until exit), so lattices above
 * WLG_NOALLOC_MAX_SITES sites are rejected.  The first call on a device looks
 * up that array's device address (cudaGetSymbolAddress); with CUDA's lazy
 * module loading that call also loads the library's module, and the array
 * with it, onto the device, which needs device memory once.  Make the first
 * call on each device at start-up, before a preallocated arena claims the
 * memory and before any stream capture.  links and out must live on the
 * current device (or be managed memory); a pointer into another GPU's memory
 * is rejected.  All calls share the array: calls that overlap
 * on the GPU race and must not be issued.  It calls no cudaMalloc, cudaFree
 * or other allocating routine. */
#define WLG_NOALLOC_MAX_SITES 33554432
int wlg_plaq_sum_noalloc(const double* links, const int n[4], int bc, double* out, void* stream);

/* ---- kernel timing (CUDA events on the context's stream) ------------------ */
int wlg_set_profiling(wlg_ctx* ctx, int on);
/* name: "hyp", "ape", "plaq", "lines", "contract", "reduce" */
int wlg_kernel_time(wlg_ctx* ctx, const char* name, double* total_ms, long long* launches);
int wlg_reset_kernel_times(wlg_ctx* ctx);
/* Tuning knobs of the contraction kernel (0 = automatic): G bottom levels
 * per thread (1,2,3,4,6), nCB column blocks per (x0, level group), block
 * threads (multiple of 32, at most 128). */
int wlg_set_contract_shape(wlg_ctx* ctx, int G, int nCB, int block);
/* As above plus the kernel form (2: register-prefetching, 3: staged top
 * lines, shuffle reduction; 4: staged top lines, shared-memory reduction;
 * 5: form 4 with its level loops unrolled for msl 4-6; 6 / 7: forms 5 / 4
 * with the top lines staged by bulk copies; 8: form 5 with the FP32
 * products as packed two-lane FMAs and the staged lines read one level
 * ahead, FP32 contexts only, an FP64 context runs form 5; 9: form 8 with one
 * 32-column chunk per warp, 72-byte line staging and per-warp partial
 * records, for four blocks per SM, FP32 contexts with msl 4-6 and the
 * default G only; 10: form 8 with the signs of the packed products in the
 * shared broadcast pairs, the same result; 11: the temporal-gauge form, the
 * default) and SB top levels per reduction (1 or 2; form 3 only).
 *
 * The temporal-gauge form (11) transforms the smeared links to the gauge in
 * which the temporal lines are unit matrices (g(x0) = U0(0) ... U0(x0-1),
 * exact for links that are unitary only approximately) and evaluates every
 * loop as a dot product of two transformed lines: a banded Gram product.  It
 * is used for every measurement on lattices of at least 32768 sites unless
 * another form is asked for here (variant 11 asks for it on any lattice),
 * and it falls back to the default carried-line form (7 FP64, 10 mixed) when
 * g g^dag differs from 1 by more than 1/4 anywhere (links smeared without
 * projection) or when msl and mwlt do not fit its kernel; wlg_contract_form
 * tells which form ran.  After it the spatial lines that
 * wlg_download_lines returns are rebuilt from the level store on request. */
int wlg_set_contract_tuning(wlg_ctx* ctx, int variant, int G, int SB, int nCB, int block);
/* The contraction form the last measurement on ctx used (0: none yet). */
int wlg_contract_form(wlg_ctx* ctx, int* form);
/* Shape of the temporal-gauge form's Gram kernel (0: automatic): occ the
 * occupancy variant (1: one block of up to 256 threads per SM, 2: two of up
 * to 192, 3: one of up to 384, where a kernel exists), ord the
 * order of its FMAs (1: dot-product chains, 2: one component at a time),
 * bx an upper bound on the start slices per block, stages the copy pipeline
 * depth (2-4), cpc the column chunks per block.  Results do not depend on
 * occ, ord, bx or stages; cpc sets how the FP32 sums of the mixed form are
 * split (FP32 rounding only). */
int wlg_set_gram_tuning(wlg_ctx* ctx, int occ, int ord, int bx, int stages, int cpc);
/* The plan those settings give for msl levels and mwlt on ctx's lattice:
 * shape[10] = {extents per thread, occ, ord, start slices per block, blocks
 * of start slices, stages, chunks per block, column splits, threads per
 * block, shared memory per block in KiB}. */
int wlg_gram_shape(wlg_ctx* ctx, int msl, int mwlt, int* shape);
/* The same plan without a context or a GPU (the SM count then defaults to
 * 148): n the lattice, tune {occ, ord, bx, stages, cpc} or NULL; shape[16] =
 * {extents per thread, occ, ord, start slices per block, its rows padded to
 * 8, extent groups, B rows per level, padded to 8, blocks of start slices,
 * staged rows, stages, threads per block, shared memory bytes per block,
 * column chunks, chunks per block, column splits}.  Lattices and boundary
 * conditions that wlg_create refuses are refused here too; -1 also when no
 * plan fits (the carried-line form then measures). */
int wlg_gram_plan_shape(const int n[4], int bc, int msl, int mwlt, int precision,
                        const int tune[5], long long shape[16]);
/* The context's CUDA stream (cudaStream_t), for callers that record events. */
void* wlg_stream(wlg_ctx* ctx);
/* Number of wloop_b200 kernel launches issued by this process so far. */
long long wlg_launch_count(void);
/* Keep a device copy of the current gauge field / put it back (device to
 * device; lets repeated measurements start from the unsmeared field). */
int wlg_snapshot(wlg_ctx* ctx);
int wlg_restore(wlg_ctx* ctx);
/* Symmetries of the measurement, for invariance checks at full size
 * (devel/wloop/check2.c, devel/wloop/check3.c; openQCD's transform_ud and
 * shift_ud).  wlg_gauge_transform: U_mu(x) <- g(x) U_mu(x) g(x+mu)^dag on the
 * context's gauge field, g(x) a synthetic SU(3) field from (seed, eps) as in
 * wlg_generate.  wlg_shift_links: U(x) <- U(x - s), periodic; with open
 * boundary conditions only s[0] = 0 (mod N0) is accepted.  Wilson loops are
 * unchanged by the first and move to W(x0 - s0) under the second. */
int wlg_gauge_transform(wlg_ctx* ctx, uint64_t seed, double eps);
int wlg_shift_links(wlg_ctx* ctx, const int s[4]);
/* Self-test of the contraction's bounded wait for its staged lines: a
 * one-warp kernel waits for a copy that never comes, with the given limit
 * (0 < limit_s <= 10); *timed_out = 1 and the elapsed time show that the wait
 * ends by itself and reports instead of hanging. */
int wlg_selftest_wait(int device, double limit_s, int* timed_out, double* elapsed_s);
/* Achievable vector FMA throughput of the device in TFLOP/s (2 flops per
 * FMA), FP64 or FP32 (precision WLG_FP64 / WLG_MIXED), or FP32 through the
 * packed two-lane FMA fma.rn.f32x2 (WLG_PEAK_F32X2, 2 FMAs per lane and
 * instruction). */
#define WLG_PEAK_F32X2 2
int wlg_peak_flops(int precision, int device, double* tflops);

/* ---- measurement output files (host only) -----------------------------------
 * .dat of the measurement program (main/ms10.c:86-190): head = 5 int32
 * {wls, msl, mwlt, mwlr, tmax}, then per configuration int32 nc and wls
 * doubles (wl_mat, index wl_idx), little-endian.  These replace ms10's static
 * write_file_head / check_file_head / write_data / read_data.  Errors return
 * -1 with the message in wlg_dat_error(). */
const char* wlg_dat_error(void);
/* head of a measurement with parameters p on a lattice of time extent n0 */
int wlg_dat_head(const wlg_wloop_parms* p, int n0, int head[5]);
int wlg_dat_write_head(const char* path, const int head[5]);   /* creates / truncates */
int wlg_dat_check_head(const char* path, const int head[5]);
int wlg_dat_append(const char* path, int nc, const double* wl_mat, int wls);
/* complete records in the file (head copied out); -1 on a torn last record */
long long wlg_dat_count(const char* path, int head[5]);
int wlg_dat_read(const char* path, long long rec, int* nc, double* wl_mat, int wls);
/* wloop part of the .par file (wloop_parms.c:343-382): appended to path /
 * compared with the record at byte offset `offset`. */
int wlg_par_write_wloop(const char* path, const wlg_wloop_parms* p);
int wlg_par_check_wloop(const char* path, long long offset, const wlg_wloop_parms* p);
/* boundary-condition part of the .par file, which ms10 writes before the
 * wloop part (main/ms10.c:290-295, openQCD-1.4's write_bc_parms /
 * check_bc_parms): int32 bc type, then 10 doubles {cG, cG', cF, cF',
 * phi[3], phi'[3]} = {1, 1, 1, 1, 0, ...} for bc 0 (open) and 3 (periodic).
 * The record is restated from openQCD's published format (openQCD is not
 * vendored with the reference), 84 bytes. */
int wlg_par_write_bc(const char* path, int bc);
int wlg_par_check_bc(const char* path, long long offset, int bc);

/* ---- gauge configurations in openQCD's exported format (host only) ---------
 * What ms10 reads with import_cnfg (main/ms10.c:709-718; the format belongs
 * to openQCD, which the reference does not include): 4 int32 extents, one
 * double (the writer's average plaquette), then for every odd point in
 * lexicographic order the 8 links U(x,0), U(x-0,0), ..., U(x,3), U(x-3,3) as
 * su3_dble, little-endian.  links: [V][4][18] doubles, lexicographic sites.
 * These file-level calls pass the plaquette through as stored; the context
 * calls below recompute it.  Errors return -1 with the message in
 * wlg_cnfg_error(). */
const char* wlg_cnfg_error(void);
int wlg_cnfg_read_head(const char* path, int n[4], double* plaq);
int wlg_cnfg_import(const char* path, const int n[4], double* links, double* plaq);
int wlg_cnfg_export(const char* path, const int n[4], const double* links, double plaq);
/* import_cnfg into a context (main/ms10.c:709-718): reads the file (its
 * extents must be the context's), zeroes the time links of the last slice
 * with open bc (set_bc), uploads the field and recomputes the average
 * plaquette on the device in FP64 from the uploaded su3_dble links: the sum
 * of Re tr U(p) over 6 V plaquettes, or (6 N0 - 3) N1 N2 N3 with open bc.  It
 * must agree with the value in the file's head within sqrt(nplaq)
 * DBL_EPSILON, the check openQCD's import_cnfg makes; otherwise -1 with
 * "Incorrect average plaquette" (wlg_last_error).  plaq (may be NULL) gets
 * the recomputed value.  wlg_export_cnfg writes the context's field with its
 * recomputed average plaquette in the head (mixed contexts: the FP32 links
 * widened to FP64). */
int wlg_import_cnfg(wlg_ctx* ctx, const char* path, double* plaq);
int wlg_export_cnfg(wlg_ctx* ctx, const char* path, double* plaq);

#ifdef __cplusplus
}
#endif
#endif
