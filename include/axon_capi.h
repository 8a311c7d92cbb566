/*
 * axon_capi.h - C ABI of the B200 AXON engine (libaxon_b200.so).
 *
 * rakib-nyc/axon has no library API: its boundary is the `build/axon key=value` CLI
 * (src/axon.mm:660-735) and the lines it prints. Internally every stage is one Metal
 * dispatch bound to fixed buffer slots and a 26-word Params block (src/axon.mm:56-83,
 * 650-652). This header exposes the same state machine as plain C entry points so the
 * engine's own CLI (the drop-in for build/axon), tests and other hosts can drive it:
 * each function below names the reference routine it replaces.
 *
 * Conventions: all arrays are host memory owned by the caller and copied by the call;
 * sizes are element counts of uint32_t unless stated. No call exits the process: every
 * failure is an axon_status. One host thread per axon_net at a time.
 */
#ifndef AXON_CAPI_H
#define AXON_CAPI_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum axon_status {
  AXON_OK = 0,
  AXON_EINVAL = 1,   /* bad argument or configuration */
  AXON_ENOMEM = 2,   /* device or pinned host allocation failed */
  AXON_ECUDA = 3,    /* a CUDA runtime call failed */
  AXON_ETIMEOUT = 4, /* a grid-wide wait in a persistent kernel gave up; the kernel exited */
  AXON_ESTATE = 5    /* call out of order (e.g. present before init) */
} axon_status;

/* Network configuration. Field meaning and reference defaults follow the CLI keys of
 * src/axon.mm:688-735 (key name in brackets). `bandhi` is the key value: the engine
 * applies it only when `contrast` != 0, as src/axon.mm:812 does. */
typedef struct axon_cfg {
  uint32_t ncol;          /* [ncol] columns of 32 neurons, multiple of 32, <= 8192 */
  uint32_t incols;        /* [incols] clamped input columns */
  uint32_t inbr;          /* [inbr] afferent branches of 32 */
  uint32_t nand;          /* [nand] initial functional density 2^-nand */
  uint32_t target;        /* [target] active columns (top-K) */
  uint32_t k;             /* [k] winners per column */
  uint32_t ktest;         /* [ktest] readout-only k override, 0 = k */
  uint32_t dthr;          /* [dthr] dendritic branch threshold */
  uint32_t boost;         /* [boost] supralinear NMDA bonus */
  uint32_t mode;          /* [mode] 0 point, 1 supralinear, 2 two-layer */
  uint32_t biasup;        /* [biasup] already resolved (1 = auto is resolved by the caller) */
  uint32_t biasdown;      /* [biasdown] */
  uint32_t biasshift;     /* [biasshift] */
  uint32_t biasdownevery; /* [biasdownevery] */
  uint32_t bandlo;        /* [bandlo] */
  uint32_t bandhi;        /* [bandhi] */
  uint32_t contrast;      /* [contrast] contrastive clamped/free phases */
  uint32_t margingate;    /* [margingate] */
  uint32_t hetero;        /* [hetero] */
  uint32_t ltdrep;        /* [ltdrep] */
  uint32_t ltdevery;      /* [ltdevery] >= 1 when contrast != 0 */
  uint32_t facil;         /* [facil] readout-only facilitation */
  uint32_t topkpar;       /* [topkpar] 1 = k_topk_par semantics, 0 = k_topk_serial */
  uint32_t reserved[9];   /* zero */
} axon_cfg;

/* Fills `cfg` with the reference's built-in defaults (not config C). */
void axon_cfg_defaults(axon_cfg* cfg);

typedef struct axon_net axon_net;

/* Device buffers of one network, named after the reference's MTLBuffers
 * (src/axon.mm:749-768). Sizes in uint32 words for ncol columns, N = 32*ncol. */
typedef enum axon_buf {
  AXON_BUF_W0 = 0, AXON_BUF_W1 = 1, AXON_BUF_W2 = 2, AXON_BUF_W3 = 3, /* ncol*32*2*32*4 each */
  AXON_BUF_CONN = 4,      /* ncol*32 : branch -> presynaptic group */
  AXON_BUF_SPK_A = 5,     /* ncol : spike ballots, written on odd steps */
  AXON_BUF_SPK_B = 6,     /* ncol : spike ballots, written on even steps */
  AXON_BUF_DRIVE = 7,     /* ncol : column drive of the last step */
  AXON_BUF_BBITS = 8,     /* N : branch-NMDA masks of the last step */
  AXON_BUF_ACC = 9,       /* N : per-neuron drive of the last step */
  AXON_BUF_BIAS = 10,     /* N : intrinsic bias */
  AXON_BUF_MARG = 11,     /* ncol : k/(k+1) margin flag of the last step */
  AXON_BUF_REFBALL = 12,  /* ncol : reference assembly whose members' drive is logged */
  AXON_BUF_DRIVELOG = 13, /* 256 : 4 words per step (shared sum, count, exclusive sum, count) */
  AXON_BUF_MULT = 14,     /* N : assembly multiplicity per neuron */
  AXON_BUF_STIM = 15,     /* ncol : input clamp pattern of the last present */
  AXON_BUF_STATS = 16,    /* 1024 : activity/plasticity counters of the last present */
  AXON_BUF_HIST = 17,     /* 64*ncol : per-step spike ballots of the last present */
  AXON_BUF_THETA = 18     /* 16 : [0] column threshold of the last step */
} axon_buf;

/* Allocates all device state of one network on `device` (0-based). Replaces the buffer
 * allocation of src/axon.mm:749-768. */
axon_status axon_create(const axon_cfg* cfg, int device, axon_net** out);
axon_status axon_destroy(axon_net* net);

/* Seeded weight-plane and connectivity init: k_init_w + k_init_conn, src/axon.mm:86-117,
 * dispatched at src/axon.mm:770-781. Also zeroes bias, theta and stats. */
axon_status axon_init(axon_net* net, uint32_t seed);

/* One presentation: present(), src/axon.mm:815-888. `stim` is the ncol-word clamp
 * pattern loadStim() builds (0 or 0xFFFFFFFF per input column). T steps in one
 * persistent launch. use_bias: 0 off, 1 on, 2 = on while learning (the reference's
 * default). Writes wall milliseconds per step to *ms_per_step when non-NULL. */
axon_status axon_present(axon_net* net, const uint32_t* stim, uint32_t T, uint32_t clamp_steps,
                         int learn, int freeze, uint32_t use_bias, double* ms_per_step);

/* Copies a device buffer to / from host memory (`words` must equal the buffer size).
 * Replaces the reference host's direct reads of shared MTLBuffer contents. */
axon_status axon_read(axon_net* net, axon_buf which, uint32_t* host, uint64_t words);
axon_status axon_write(axon_net* net, axon_buf which, const uint32_t* host, uint64_t words);
uint64_t axon_buf_words(const axon_net* net, axon_buf which);

/* Functional synapse count: k_wstat, src/axon.mm:641-646 (u32 wrap-around total). */
axon_status axon_wstat(axon_net* net, uint32_t* count);

/* Within-assembly functional density counters: k_within, src/axon.mm:524-562.
 * out[10] (u32, added to by the call as the reference's atomics do; pass zeros).
 * post_mask is read only when use_mask != 0 (N words); mult is N words or NULL (zeros). */
axon_status axon_within(axon_net* net, const uint32_t* ball, uint32_t use_mask,
                        const uint32_t* post_mask, const uint32_t* mult, uint32_t out[10]);

/* Per-neuron functional in-degree over recurrent branches: k_indeg, src/axon.mm:566-581. */
axon_status axon_indeg(axon_net* net, uint32_t* out_n);
/* Per-neuron count of recurrent synapses still at 5 or 6: k_untouched, src/axon.mm:501-519. */
axon_status axon_untouched(axon_net* net, uint32_t* out_n);
/* Counter histogram: k_wdiag, src/axon.mm:591-638. memb N words, asm_spk nstim*ncol
 * words, hist48 accumulated. */
axon_status axon_wdiag(axon_net* net, const uint32_t* memb, const uint32_t* asm_spk,
                       uint32_t nstim, uint32_t sel, uint32_t hist48[48]);
/* Bit-serial known-answer hook: k_bstest, src/axon.mm:424-434. a0..a3 and m hold n
 * words each (n a multiple of 4); op 0 inc, 1 dec, 2 clip [lo,hi]; planes updated. */
axon_status axon_bstest(int device, uint32_t op, uint32_t lo, uint32_t hi, uint32_t* a0,
                        uint32_t* a1, uint32_t* a2, uint32_t* a3, const uint32_t* m, uint64_t n);
/* k-of-32 known-answer hook: the kernels' exact k-WTA ranking (kwta_ballot_margin,
 * src/axon.mm:134-144) on n columns: v holds 32 values per column, k one k per column;
 * out receives per column the winners ballot, vk and vk1 (3 words). */
axon_status axon_kwtatest(int device, const uint32_t* v, const uint32_t* k, uint32_t* out, uint32_t n);

/* Stimulus patterns: `nstim` rows of `stimcols` input-column indices, drawn as
 * src/axon.mm:793-799 does (mt19937(7 + seed*104729), libc++ shuffle of 0..incols-1). */
axon_status axon_stimuli(uint32_t seed, uint32_t nstim, uint32_t incols, uint32_t stimcols, uint32_t* out);
/* Clamp pattern of one presentation: loadStim, src/axon.mm:800-804. Keeps each of the
 * `ncols` pattern columns with probability `keep` (mt19937(seed), tested in order). */
axon_status axon_load_stim(const uint32_t* cols, uint32_t ncols, double keep, uint32_t seed, uint32_t ncol,
                           uint32_t* out_ncol);

/* Noisy cue: no counterpart in the reference, whose cues only drop whole pattern columns
 * (loadStim's keep fraction, src/axon.mm:800-804). Clamp words of the whole pattern
 * (`ncols` distinct columns, each < ncol, all 32 neurons on), then round(frac * A) of its
 * A = 32 * ncols active bits flipped off: the active bits are listed column by column in
 * `cols` order, bit 0 first, and the flipped ones are the first round(frac * A) picks of
 * a forward Fisher-Yates over that list driven by mt19937(seed), pick i drawn from
 * [i, A-1] as the shuffle of axon_stimuli draws. frac in [0, 1]. */
axon_status axon_noisy_cue(const uint32_t* cols, uint32_t ncols, double frac, uint32_t seed, uint32_t ncol,
                           uint32_t* out_ncol);
/* The seed of draw `draw` of pattern q's noisy cue at `pct` percent of active bits
 * flipped, as the CLI's cueflip row and the batched-recall benchmark use it:
 * 90000 + 1000*pct + 16*q + draw. */
uint32_t axon_noisy_cue_seed(uint32_t q, uint32_t pct, uint32_t draw);

/* ---------------------------------------------------------------- batched readout
 * B readout trajectories of one network, each exactly what present() with learn = 0 does
 * (src/axon.mm:815-888): `cues` holds B clamp patterns of ncol words, of which only the
 * first incols (the input columns the clamp sets) are read, and axon_recall copies only
 * those to the device. The batched method
 * runs all B in one launch that reads each W3 tile once for every trajectory; the plain
 * method runs them one presentation at a time (same results, for comparison). Outputs
 * are optional (NULL to skip): final_spk B*ncol spikes of the last step, hist B*T*ncol
 * spikes of every step, stats B*1024 counters of k_emit (word 2, the branch-coincidence
 * count, is produced by the plain method only), drive_log B*256 added to like the
 * reference's driveLog buffer for the members marked in ref_ball (B*ncol, NULL = none;
 * the shared/exclusive split uses the network's MULT buffer). gpu_ms receives the
 * device time of the launches. The network's per-present buffers are left undefined. */
typedef enum axon_recall_method { AXON_RECALL_BATCHED = 0, AXON_RECALL_PLAIN = 1 } axon_recall_method;

typedef struct axon_recall_args {
  uint32_t T;           /* steps per trajectory, 1..64; up to 1024 for the batched method when
                           hist, stats, drive_log and ref_ball are all NULL */
  uint32_t clamp_steps; /* leading steps clamped to the cue */
  uint32_t use_bias;    /* 0 off (the reference's readout default), 1 on */
  uint32_t method;      /* axon_recall_method */
  uint32_t graph;       /* batched method: 1 = run the launch(es) and their buffer resets as a
                           captured CUDA graph, kept and replayed while every argument and
                           array stays the same (device-resident callers); 0 = launch directly */
  uint32_t contraction; /* batched method: the unit that computes k_drive's AND-popcounts
                           (src/axon.mm:166-173): AXON_CONTRACT_POPC (0, __popc on the CUDA
                           cores) or AXON_CONTRACT_TENSOR (1, binary MMA on the tensor cores);
                           the results are the same */
  uint32_t slab;        /* batched method, 16-bit counters without bias or facilitation: which
                           per-neuron drives the kernel stores for the k-of-32 of the columns
                           that pass the gate. AXON_SLAB_FLOOR (0): those of columns whose
                           drive reaches the trajectory's threshold-histogram floor (half its
                           previous threshold), and every one at the step after the clamp;
                           AXON_SLAB_FLOOR_ALWAYS (1): the floor at every step; AXON_SLAB_FULL
                           (2): every one. A gated column without a stored drive has it
                           recomputed; the results are the same */
  uint32_t reserved[1]; /* zero */
} axon_recall_args;

enum { AXON_CONTRACT_POPC = 0, AXON_CONTRACT_TENSOR = 1 };
enum { AXON_SLAB_FLOOR = 0, AXON_SLAB_FLOOR_ALWAYS = 1, AXON_SLAB_FULL = 2 };

axon_status axon_recall(axon_net* net, const uint32_t* cues, uint32_t B, const axon_recall_args* args,
                        const uint32_t* ref_ball, uint32_t* final_spk, uint32_t* hist, uint32_t* stats,
                        uint32_t* drive_log, double* gpu_ms);
/* As axon_recall, with every array in device memory of the network's GPU (no copies). */
axon_status axon_recall_device(axon_net* net, const uint32_t* cues, uint32_t B, const axon_recall_args* args,
                               const uint32_t* ref_ball, uint32_t* final_spk, uint32_t* hist, uint32_t* stats,
                               uint32_t* drive_log, double* gpu_ms);

/* ---------------------------------------------------------------- allocation-free present
 * No counterpart in the reference. For hosts that must not allocate device memory during
 * a call (their own caching allocator owns the device, or allocation is forbidden after
 * start-up): the same presentation as axon_present, run on buffers the caller already
 * owns, passed as device pointers with the sizes listed for axon_buf (plus stim: ncol
 * words, the clamp pattern). Allocates nothing - no cudaMalloc/cudaFree, no library
 * allocation: the kernel's only scratch is a fixed device array in the library sized for
 * ncol <= 4096 (about 87 KiB per GPU, held until the process exits); larger ncol returns
 * AXON_EINVAL. Every pointer must be 16-byte aligned (the planes are read as 16-byte
 * vectors and W3 tiles are bulk-copied); a misaligned one returns AXON_EINVAL. The call is
 * synchronous on the legacy default stream: it returns when the presentation is done, and
 * must not be made while any stream of the device is being captured. The first call on a
 * device resolves the array's device address and keeps it for the process, so the library
 * must not outlive a cudaDeviceReset of that device. Calls that overlap on the GPU share
 * that array and race: issue one at a time per device. */
typedef struct axon_state_dev {
  uint32_t *w0, *w1, *w2, *w3;                   /* bitplanes (in/out) */
  uint32_t *conn, *bias, *mult, *refball, *stim; /* conn, mult, refball, stim in; bias in/out */
  uint32_t *spk_a, *spk_b, *drive, *bbits, *acc, *marg, *drive_log, *stats, *hist, *theta; /* out */
} axon_state_dev;

axon_status axon_present_static(const axon_cfg* cfg, const axon_state_dev* state, uint32_t T,
                                uint32_t clamp_steps, int learn, uint32_t use_bias);

/* ---------------------------------------------------------------- checkpoints
 * The reference keeps no trained network: each run retrains from the seed
 * (src/axon.mm:1001-1033). A checkpoint file holds one network's trained state - the
 * W0..W3 planes, conn, bias and mult (the MTLBuffers of src/axon.mm:749-768) - with its
 * axon_cfg and the caller's training metadata, each section and the whole file under an
 * FNV-1a-64 checksum. axon_load verifies magic, version, configuration (it must equal the
 * network's) and checksums before it changes the network; on success the network is
 * initialised, its stats and theta cleared. */
typedef struct axon_ckpt_meta {
  uint32_t seed;        /* [seed] the network and its patterns were made from */
  uint32_t nstim;       /* [stim] patterns stored (the load) */
  uint32_t stimcols;    /* [stimcols] columns per pattern */
  uint32_t epochs;      /* [epochs] trained */
  uint32_t reserved[4]; /* zero */
} axon_ckpt_meta;

axon_status axon_save(axon_net* net, const char* path, const axon_ckpt_meta* meta);
axon_status axon_load(axon_net* net, const char* path, axon_ckpt_meta* meta_out);

/* ---------------------------------------------------------------- many networks, one launch
 * The reference trains and reads out one network per process: build/axon runs init,
 * epochs x nstim learning presentations plus one more of pattern 0 (src/axon.mm:1001-1033),
 * then the readouts its measurements come from (src/axon.mm:1080-1105, 1495-1508,
 * 1695-1730, 1804-1858). axon_multi_train runs that experiment for n networks at once:
 * every network is initialised from seeds[i] with nstim[i] patterns (its load) and all
 * their presentations run inside ONE persistent launch (captured as a CUDA graph when
 * args->graph != 0), in slots of SMs that each take a queue of networks. The networks
 * must share one axon_cfg and one device. With autotune != 0 the slot count and CTA shape
 * are chosen by timing candidates on the networks themselves (they are re-initialised
 * afterwards); networks are assigned to slots longest-first. method = 1 runs the same
 * presentations through the plain path instead (one present launch each), for
 * comparison. The ten settle presentations of src/axon.mm:1001 are not run: they change
 * no weight or bias. With readout != 0, results[i] holds network i's measurements,
 * computed as the reference's printing blocks compute them. */
typedef struct axon_multi_args {
  uint32_t epochs;      /* [epochs] */
  uint32_t T;           /* [T] steps per presentation, 1..64 */
  uint32_t clamp_steps; /* [clampsteps] cue steps of the readouts */
  uint32_t train_clamp; /* [trainclamp] clamped steps of a learning presentation */
  uint32_t stimcols;    /* [stimcols] columns per pattern */
  uint32_t wave_t;      /* [wavet] steps of the wave readout (at most 60 are run) */
  uint32_t readout;     /* 1: run the readouts and fill results */
  uint32_t autotune;    /* 1: pick slots and CTA shape by timing candidates */
  uint32_t slots;       /* autotune == 0: concurrent networks (0 = one per network, at most one per SM) */
  uint32_t threads;     /* autotune == 0: 1024 or 896 (4 W3 tiles in flight per warp) or 512 (8 tiles) */
  uint32_t graph;       /* 1: launch through a captured CUDA graph */
  uint32_t method;      /* 0: one persistent launch, 1: plain path, one launch per presentation */
  uint32_t reserved[4]; /* zero */
} axon_multi_args;

typedef struct axon_multi_result {
  double within_pct; /* "within-assembly : ... = X%" (deep block) */
  double recall;     /* 75% cue row: mean overlap with the own clamped reference */
  double best_other; /* 75% cue row: mean best overlap with another reference */
  double drive_t6;   /* "t6:" free-phase drive to assembly members */
  double wave_first; /* wave ov(clampRef) at the first free step */
  double wave_last;  /* wave ov(clampRef) at the last step (sustained = last / first, as printed) */
  double wdens_pct;  /* functional synapse density after training, % */
  uint64_t steps;    /* steps this network ran */
} axon_multi_result;

typedef struct axon_multi_report {
  double gpu_ms;        /* device time of the training + readout launch (or of all plain launches) */
  double tune_ms;       /* device time spent timing candidate shapes */
  uint64_t steps;       /* network-steps run */
  uint64_t train_steps; /* of which learning steps */
  uint32_t slots, threads, tiles, grid; /* shape used (slots = 0 for the plain path) */
  uint32_t graph;       /* 1 when the launch ran as a CUDA graph */
  uint32_t tried;       /* candidate shapes timed */
  uint64_t w3_tiles;    /* W3 tiles (1 KiB each) the drive read: (column, branch) pairs with a spiking group */
  uint64_t learn_tasks; /* branch updates of k_learn (W0..W3 tiles read and written, 8 KiB each) */
} axon_multi_report;

axon_status axon_multi_train(axon_net* const* nets, uint32_t n, const uint32_t* seeds, const uint32_t* nstim,
                             const axon_multi_args* args, axon_multi_result* results, axon_multi_report* report);

/* ---------------------------------------------------------------- recall serving
 * The reference runs one readout at a time: present() with learn = 0 (src/axon.mm:815-888),
 * the clamp built from a pattern's kept columns (src/axon.mm:800-804). A server answers
 * such readouts as requests against device-resident trained networks, with continuous
 * batching: an internal thread advances, tick by tick, every admitted trajectory by one
 * step in one batched pass (trajectories of one network share each weight-tile load),
 * admits requests that have arrived into slots as they free up (the slot count follows
 * from mem_bytes, the device memory the server may use), and retires finished ones. A
 * request's final spikes are the same as those of axon_recall for the same network, cue
 * and steps, whatever else is in flight. The networks must share one axon_cfg and device
 * and must not be changed (present, write, init) while the server exists.
 * Times are seconds of axon_clock_s(), a monotonic host clock. */
typedef struct axon_server axon_server;

typedef struct axon_serve_result {
  uint64_t tag;    /* the caller's request id */
  uint32_t net;    /* network index */
  uint32_t steps;  /* clamped + free steps run */
  double arrive_s; /* arrival time given at submission */
  double admit_s;  /* time the request got a slot */
  double done_s;   /* time its final spikes reached the host */
} axon_serve_result;

typedef struct axon_serve_counters {
  uint32_t slots;      /* trajectory slots the memory budget allows */
  uint32_t in_flight;  /* slots in use now */
  uint64_t queued;     /* submitted, not yet admitted */
  uint64_t ticks;      /* batched steps run */
  uint64_t completed;  /* requests finished */
  uint64_t max_batch;  /* most trajectories advanced in one tick */
  double mean_batch;   /* trajectories per tick, mean */
  double busy_s;       /* time spent in ticks */
  double drive_s;      /* device time of the drive kernel, summed over ticks */
  double emit_s;       /* device time of the threshold/emit kernel, summed over ticks */
  uint64_t slot_bytes; /* device memory one trajectory slot takes */
  uint64_t fixed_bytes;/* device memory of the server besides its slots: slots = (mem_bytes - fixed) / slot */
} axon_serve_counters;

double axon_clock_s(void);
axon_status axon_serve_create(axon_net* const* nets, uint32_t n, uint64_t mem_bytes, axon_server** out);
/* cue_cols: the ncue input columns clamped on (each < incols); the trajectory runs
 * clamp_steps clamped then free_steps free steps. arrive_s: arrival time (0 = now); a
 * request is not admitted before it. Latency = done_s - arrive_s. */
axon_status axon_serve_submit(axon_server* s, uint32_t net, const uint32_t* cue_cols, uint32_t ncue,
                              uint32_t clamp_steps, uint32_t free_steps, uint64_t tag, double arrive_s);
/* Up to max_results finished requests, oldest first; final_spk (NULL to skip) receives
 * ncol words per result. */
axon_status axon_serve_poll(axon_server* s, axon_serve_result* res, uint32_t* final_spk, uint32_t max_results,
                            uint32_t* n_out);
/* Blocks until nothing is queued or in flight (AXON_ETIMEOUT after timeout_s). */
axon_status axon_serve_wait_idle(axon_server* s, double timeout_s);
axon_status axon_serve_stats(axon_server* s, axon_serve_counters* out);
axon_status axon_serve_destroy(axon_server* s);

/* A second network with the same configuration and a copy of every device buffer of
 * `src` (planes, conn, bias, mult, the per-present buffers). No counterpart in the
 * reference; the profile mode uses it so that profiling changes no network. */
axon_status axon_clone(const axon_net* src, axon_net** out);

/* profile=1 of the reference (src/axon.mm:1161-1256) times each of its five kernels with
 * Metal timestamps over one learning presentation. Here the five run fused in one
 * persistent launch, so the same presentation is timed per phase with the device timer:
 * out[0..3] = us per step of drive + k-of-32 (k_drive, the ballot of k_emit), the grid
 * barrier, threshold + gate + spike rebuild (k_topk, k_emit), records + bias + learning
 * (k_emit's counters, k_bias, k_learn), each the mean over CTAs; out[4] = us per step;
 * out[5] = the launch in ms. The presentation itself is an ordinary axon_present. */
axon_status axon_profile_present(axon_net* net, const uint32_t* stim, uint32_t T, uint32_t clamp_steps, int learn,
                                 uint32_t use_bias, double out[6]);

/* Grid-wait limit of the persistent kernels in nanoseconds (default 2e9). */
axon_status axon_set_wait_limit(axon_net* net, uint64_t ns);
/* No counterpart in the reference (it has no failure detection). Test hook for the bounded
 * waits: the next persistent launch of this network (axon_present, or axon_multi_train
 * when the network is nets[0]) waits at every grid barrier for `missing` CTAs that were
 * never launched, as if they had died. The first barrier then runs out after the wait
 * limit, every CTA returns, and the call reports AXON_ETIMEOUT; the GPU context stays
 * usable. One-shot. */
axon_status axon_inject_missing_arrival(axon_net* net, uint32_t missing);
/* Text of the last error on this thread. */
const char* axon_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* AXON_CAPI_H */
