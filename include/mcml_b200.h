/*
 * mcml_b200.h -- C ABI of the B200-native MCML photon-transport library.
 *
 * The reference (MCML_GPU K3.02) has no library boundary: its CLI, host
 * driver and kernels share one process and a set of global __constant__
 * symbols.  This header is the seam a maintainer of that code base would
 * bind to instead.  Every entry point names the reference function(s) it
 * replaces as file:line of the reference project.
 *
 * Conventions
 *  - Every call returns MCML_OK (0) or a negative mcml_status.  Nothing is
 *    printed by the library; mcml_last_error() holds a message for the
 *    calling thread.
 *  - The caller owns every struct and host array passed in.  The library
 *    owns the device buffers of an mcml_ctx and frees them in mcml_destroy.
 *  - An mcml_ctx holds one simulation's parameter block (the reference's
 *    __constant__ tables, header.h:205-214) and its device buffers.  Use
 *    one context per host thread or stream; contexts share no state.
 *  - Weights are in the reference's units: an integer number of quanta of
 *    1/0xFFFFFFFF of a launched photon, held in float (header.h:95).
 */
#ifndef MCML_B200_H
#define MCML_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Limits of the reference: PRESET_NUM_LAYER and PRESET_NUM_DETECTOR (header.h:38,44). */
#define MCML_MAX_LAYERS 10
#define MCML_MAX_SDS 30

/* Absorbance grid of the reference: record_nr/nz/dr/dz (header.h:65-68). */
#define MCML_REF_GRID_NR 1000
#define MCML_REF_GRID_NZ 500
#define MCML_REF_GRID_D 0.01f

typedef enum mcml_status {
  MCML_OK = 0,
  MCML_INCOMPLETE = 1,  /* a checkpointed run stopped early; call again */
  MCML_E_INVALID = -1,  /* bad argument or configuration value        */
  MCML_E_CUDA = -2,     /* a CUDA runtime call failed                  */
  MCML_E_NOMEM = -3,    /* host or device allocation failed            */
  MCML_E_OVERFLOW = -4, /* detection-record buffer too small           */
  MCML_E_IO = -5,       /* file could not be opened or written         */
  MCML_E_PARSE = -6,    /* sim_set.json / input.txt could not be read  */
  MCML_E_STATE = -7,    /* calls made in the wrong order               */
  MCML_E_BUDGET = -8,   /* a kernel hit its step budget and stopped    */
  MCML_E_NODEV = -9,    /* no CUDA device                              */
  MCML_E_CHECKPOINT = -10 /* checkpoint file corrupt or of another run  */
} mcml_status;

/*
 * One simulation: the fields of sim_set.json plus one line of input.txt,
 * already converted to the types the reference stores them in
 * (io.cpp:48-191 for the JSON keys, io.cpp:138-147 for input.txt).
 * Angles are in degrees, as in the file; the library converts them with
 * the reference's float arithmetic (io.cpp:184,190).
 */
typedef struct mcml_sim {
  uint64_t number_photons;      /* "number_photons"                         */
  uint32_t num_layers;          /* "number_layers" (1..MCML_MAX_LAYERS)     */
  uint32_t num_sds;             /* "probes.num_SDS" (1..MCML_MAX_SDS)       */
  float upper_n;                /* "upper_n"                                */
  float lower_n;                /* "lower_n"                                */
  float detector_reflectance;   /* "detector_reflectance" in [0,1]          */
  int32_t source_probe_oblique; /* 1: pencil beam at "angle"; 0: disc+cone  */
  int32_t detector_probe_oblique; /* 1: oblique fibre ovals; 0: rings       */
  float source_NA;
  float source_radius;          /* cm                                       */
  float source_angle_deg;
  float det_pos[MCML_MAX_SDS];       /* cm from the source centre           */
  float det_NA[MCML_MAX_SDS];
  float det_radius[MCML_MAX_SDS];    /* cm                                  */
  float det_angle_deg[MCML_MAX_SDS];
  float height[MCML_MAX_LAYERS];     /* cm; the last layer's value is unused */
  float mua[MCML_MAX_LAYERS];        /* 1/cm                                */
  float mus[MCML_MAX_LAYERS];        /* 1/cm                                */
  float n[MCML_MAX_LAYERS];
  float g[MCML_MAX_LAYERS];
} mcml_sim;

/* Run options.  Zero-initialise and set what you need. */
typedef struct mcml_opts {
  uint64_t seed;            /* XORWOW seed (reference: time(NULL), transport.cu:72) */
  uint64_t slots;           /* RNG subsequences ("photon slots"): slot s walks its
                               photons in order on subsequence s, as the reference's
                               thread s does.  0 = automatic: N when N is at most
                               the reference's thread count on this device
                               (SMs x max threads/SM, io.cpp:522-526) -- its
                               one-photon-per-thread layout, bit-exact when N equals
                               it -- else about 4 photons per slot.                  */
  int32_t device;           /* CUDA ordinal (reference: -G, main.cu:51-59)          */
  uint32_t grid_nr;         /* absorbance grid; 0 = 1000                            */
  uint32_t grid_nz;         /* 0 = 500                                              */
  float grid_dr;            /* cm; 0 = 0.01                                         */
  float grid_dz;            /* cm; 0 = 0.01                                         */
  uint64_t record_capacity; /* detection records kept on the device; 0 = automatic  */
  void *stream;             /* cudaStream_t to launch on; NULL = a library stream   */
  uint32_t block_size;      /* threads per block of the walk; 0 = tuned default     */
  uint32_t blocks_per_sm;   /* resident blocks per SM of the walk; 0 = tuned        */
  uint64_t replay_step_budget; /* max steps of one replayed photon; 0 = 1<<26        */
  uint64_t slot_begin;      /* first subsequence of this context: a shard of a
                               multi-GPU run uses slot_begin = rank * slots          */
} mcml_opts;

/* Per-SDS result of the first pass (and, after mcml_replay, of the replay). */
typedef struct mcml_result {
  uint32_t num_sds;
  uint64_t photons;                  /* photons walked                        */
  uint64_t steps;                    /* walk steps (loop iterations)          */
  uint64_t detected[MCML_MAX_SDS];   /* SDS_detected_number (io.cpp:374-378)  */
  double weight_sum[MCML_MAX_SDS];   /* sum of detected weights, in quanta     */
  double weight_sumsq[MCML_MAX_SDS]; /* sum of squared detected weights        */
  double reflectance[MCML_MAX_SDS];  /* weight_sum / (0xFFFFFFFF * N) (io.cpp:16-28) */
  double std_error[MCML_MAX_SDS];    /* standard error of reflectance[]       */
  float walk_ms;                     /* device time of the walk kernel        */
  float replay_ms;                   /* device time of the replay             */
  float seed_ms;                     /* device time of the slot seeding       */
  uint64_t slots;                    /* RNG subsequences the run used         */
} mcml_result;

typedef struct mcml_device_info {
  char name[100];
  int32_t major, minor;
  int32_t sm_count;
  int32_t max_threads_per_sm;
  uint64_t global_mem;
  uint64_t reference_threads; /* the reference's autototalthread (io.cpp:522-526) */
} mcml_device_info;

typedef struct mcml_ctx mcml_ctx;

/* ---- library ---------------------------------------------------------- */
const char *mcml_version(void);
const char *mcml_strerror(int status);
/* Message of the last failing call on this thread (never NULL). */
const char *mcml_last_error(void);

/* Replaces list_GPU (io.cpp:495-544) for one device. */
int mcml_device_count(int *count);
int mcml_get_device_info(int device, mcml_device_info *info);

/* ---- configuration ---------------------------------------------------- */
/*
 * Replaces read_mua_mus (io.cpp:35-256): reads sim_set.json and input.txt
 * into up to max_sims mcml_sim structs.  Checks the same things the
 * reference checks, with the same wording in mcml_last_error():
 * oblique flags 0/1, detector_reflectance in [0,1], layer and SDS limits,
 * detector count vs list size, and the last layer's mus>0, n>1, g<=1.
 */
int mcml_parse_config(const char *sim_json_path, const char *input_txt_path,
                      mcml_sim *sims, int max_sims, int *num_sims);

/* Derived per-simulation constants, computed exactly as io.cpp:168-238 does. */
typedef struct mcml_derived {
  float z_min[MCML_MAX_LAYERS + 2];
  float z_max[MCML_MAX_LAYERS + 2];
  float mutr[MCML_MAX_LAYERS + 2];  /* 1/(mua+mus)                       */
  float start_weight;               /* (u32)(0xffffffff*(1-R_specular))  */
  float critical_angle[MCML_MAX_SDS + 1]; /* asin(NA/upper_n), index 1..S */
  float det_angle_rad[MCML_MAX_SDS + 1];  /* index 0 = source            */
} mcml_derived;
int mcml_derive(const mcml_sim *sim, mcml_derived *out);

/* ---- simulation ------------------------------------------------------- */
/* Replaces InitMemStructs + InitDCMem (transport.cu:1002-1070). */
int mcml_create(const mcml_sim *sim, const mcml_opts *opts, mcml_ctx **ctx);
/* Uploads a new parameter block to an existing context (same limits).  A
 * simulation rejected as invalid leaves the previous one in place; if the
 * slot states cannot be allocated (MCML_E_CUDA), runs return MCML_E_STATE
 * until a later mcml_set_sim succeeds. */
int mcml_set_sim(mcml_ctx *ctx, const mcml_sim *sim);
void mcml_destroy(mcml_ctx *ctx);

/*
 * First pass: replaces LaunchPhoton_Global + the MCd launch loop +
 * calculate_reflectance (transport.cu:106-147, 299-311).  Walks all
 * photons in one persistent launch, keeps one record per detection on the
 * device and returns per-SDS counts and weight sums.  Blocks until done.
 */
int mcml_run(mcml_ctx *ctx, mcml_result *result);
/* Same work, enqueued on the context's stream without waiting. */
int mcml_launch_run(mcml_ctx *ctx);

/*
 * Replay: replaces the per-SDS MCd_replay batches and
 * calculate_reflectance_replay (transport.cu:160-222, 315-332).  Re-walks
 * every detected photon from its saved XORWOW state, producing its row
 * [weight, PL_1..PL_L, steps], per-layer interaction counts, and the A_rz /
 * A0_z tallies.  Blocks until done; result (if non-NULL) gets the replayed
 * weight sums.
 */
int mcml_replay(mcml_ctx *ctx, mcml_result *result);
int mcml_launch_replay(mcml_ctx *ctx);

/* Waits for the context's stream and fills result from the first pass. */
int mcml_get_result(mcml_ctx *ctx, mcml_result *result);

/*
 * Detected photons of one SDS (1-based sds), ordered by photon index
 * (slot-major), which is the reference's order when N equals its thread
 * count.  photon_ids / weights may be NULL.  *count gets the number of rows.
 */
int mcml_get_detections(mcml_ctx *ctx, int sds, uint64_t *photon_ids,
                        float *weights, uint64_t capacity, uint64_t *count);

/*
 * Replay rows of one SDS in the pathlength_SDS_#.bin layout (io.cpp:302-311):
 * count rows of (L+2) float32 = weight, PL_1..PL_L [cm], steps.  Same order
 * as mcml_get_detections.  interactions (may be NULL) gets count*L uint32
 * per-layer scattering-event counts, which the reference does not record.
 */
int mcml_get_rows(mcml_ctx *ctx, int sds, float *rows, uint32_t *interactions,
                  uint64_t capacity, uint64_t *count);

/*
 * Absorbance tallies after mcml_replay, in u64 weight quanta, laid out as
 * the reference's A_rz[sds][iz][ir] and A0_z[sds][iz] (transport.cu:583-588).
 * Either pointer may be NULL.
 */
int mcml_get_tallies(mcml_ctx *ctx, uint64_t *A_rz, uint64_t *A0_z);

/*
 * The last run's outputs where they lie, in device memory, for a caller that
 * combines several GPUs' runs on the GPUs (sums of the u64 tallies and a
 * gather of the rows over NCCL) instead of through host copies.  No
 * counterpart in the reference (one GPU, host collection in
 * transport.cu:274-332).  Records (and, after mcml_replay, rows) are put in
 * file order first: SDS-major, photon order within an SDS, detected[s]
 * entries for SDS s+1.  A record is 40 bytes: photon index u64, SDS u32,
 * detected weight f32, the photon's XORWOW start state 6 x u32.  Rows are
 * row_len = L+2 float32 in the pathlength_SDS_#.bin layout.  A_rz / A0_z are
 * the u64 quanta of mcml_get_tallies.  Without a replay rows, A_rz and A0_z
 * are NULL.  The pointers belong to the context: valid until its next run,
 * replay, mcml_set_sim or mcml_destroy; work on them must be ordered after
 * `stream` (the context's stream).  Synchronises that stream.
 */
typedef struct mcml_device_outputs {
  const void *records;
  const float *rows;
  const uint64_t *A_rz;
  const uint64_t *A0_z;
  uint64_t n_records;
  uint64_t detected[MCML_MAX_SDS];
  uint64_t arz_count, a0z_count;
  uint64_t photons;
  uint32_t row_len;
  void *stream;
} mcml_device_outputs;
int mcml_get_device_outputs(mcml_ctx *ctx, mcml_device_outputs *out);

/* Replaces calculate_average_pathlength (transport.cu:274-297): out[S*L]. */
int mcml_average_pathlength(mcml_ctx *ctx, double *out);

/*
 * Writes the reference's output files for one simulation, with the
 * reference's names, modes and byte layouts (io.cpp:11-33, 281-469):
 * output_txt (append), summary.json (append), and with replay,
 * pathlength_SDS_#.{bin,txt}, average_pathlength.txt, A_rz_SDS_#.{bin,txt},
 * A0_z_SDS_#.{bin,txt}, into directory dir ("" = current directory).
 * flags: MCML_OUT_* below.  sim_s / replay_s go into summary.json.
 */
#define MCML_OUT_REPLAY 1u       /* -R  */
#define MCML_OUT_ABSORBANCE 2u   /* -A  */
#define MCML_OUT_PATHLENGTH 4u   /* -P  */
#define MCML_OUT_AVERAGE_PL 8u   /* -AP */
#define MCML_OUT_BINARY 16u      /* -B  */
int mcml_write_outputs(mcml_ctx *ctx, const char *dir, const char *output_txt,
                       uint32_t flags, double sim_s, double replay_s);

/* ---- batches of parameter sets ---------------------------------------- */
/*
 * Many tissue parameter sets in one persistent launch.  Replaces running
 * the reference once per set (its multi-simulation mode shares one
 * critical-angle table, io.cpp:193-197).  Set b (sims[b], with its own
 * number_photons) walks on ceil(N_b / photons_per_slot) slots of seed
 * seed + b -- the same photons as mcml_run on that set alone with that
 * seed and slot count, so per-set results are identical.  All sets need
 * the same source/detector modes.  The seeding and the walk are captured
 * into a CUDA graph on the first run and relaunched afterwards.  Results:
 * one mcml_result per set (counts, FP64 weight sums, reflectance and its
 * standard error; no replay).
 */
typedef struct mcml_batch_opts {
  uint64_t seed;              /* set b uses seed + b                          */
  int32_t device;
  uint32_t photons_per_slot;  /* 0 = 64                                       */
  uint32_t block_size;        /* 0 = default walk variant                     */
  uint32_t blocks_per_sm;
  void *stream;               /* NULL = a library stream (graphs cannot be
                                 captured on the legacy default stream)      */
  int32_t no_graph;           /* 1: plain launches instead of a CUDA graph    */
} mcml_batch_opts;

typedef struct mcml_batch_tuning {
  uint32_t block_size;
  uint32_t blocks_per_sm;
  uint32_t photons_per_slot;
  float pilot_ms;
} mcml_batch_tuning;

typedef struct mcml_batch mcml_batch;
int mcml_batch_create(const mcml_sim *sims, int num_sets, const mcml_batch_opts *opts,
                      mcml_batch **batch);
/* Times pilot runs (photon_fraction of each set's photons) over the walk
 * variants and photons-per-slot choices and keeps the fastest. */
int mcml_batch_autotune(mcml_batch *batch, double photon_fraction, mcml_batch_tuning *chosen);
int mcml_batch_run(mcml_batch *batch, mcml_result *results);
int mcml_batch_launch(mcml_batch *batch);
int mcml_batch_get_results(mcml_batch *batch, mcml_result *results);
void mcml_batch_destroy(mcml_batch *batch);

/* ---- White Monte Carlo relabelling ------------------------------------ */
/*
 * Reflectance of one SDS under other absorption / scattering coefficients,
 * from one replay: each combo c gives
 *   R_c = sum_i w_i prod_l (mus'_l/mus_l)^n_il exp(-sum_l (dmua_l+dmus_l) PL_il) / scale
 * over the SDS's replayed photons i (weight w, pathlengths PL, interaction
 * counts n from mcml_get_rows).  The mua-only case is the factor of
 * calculate_average_pathlength (transport.cu:285-292); the mus factor
 * needs the interaction counts the reference does not record.
 * All arrays are DEVICE pointers; work is enqueued on `stream`.
 */
typedef struct mcml_wmc_set {
  const float *pathlength;   /* L x D, layer-major: PL of photon i in layer l at [l*D+i] */
  const float *interactions; /* L x D, layer-major, interaction counts as float       */
  const float *weight;       /* D detected weights (quanta)                            */
  uint64_t count;            /* D                                                      */
  uint32_t num_layers;       /* L                                                      */
} mcml_wmc_set;
uint64_t mcml_wmc_workspace_bytes(uint64_t num_photons, uint64_t num_combos);
/* base_mua/base_mus: HOST, L each (the replayed run's coefficients).
 * combos: C x 2L (mua'_1..L, mus'_1..L).  scale: 0xFFFFFFFF * N of the run.
 * out: C doubles.  workspace: mcml_wmc_workspace_bytes(D, C) device bytes. */
int mcml_wmc_rescale(const mcml_wmc_set *set, const float *base_mua, const float *base_mus,
                     const float *combos, uint64_t num_combos, double scale, double *out,
                     void *workspace, uint64_t workspace_bytes, void *stream);

/* ---- MLP surrogate ----------------------------------------------------- */
/*
 * No counterpart in the reference.  An ensemble of MLPs
 * (in -> hidden x depth, GELU -> out) trained and evaluated by this
 * library's BF16 tensor-core kernels with FP32 accumulation and FP32
 * master weights (Adam), forward and backward products on tcgen05
 * (accumulators in tensor memory; the output layer's 3-wide input
 * gradient on the CUDA cores).  Limits: in_dim and
 * hidden at most 256, hidden a multiple of 16, out_dim <= hidden.  Inputs and targets are normalised with
 * mcml_mlp_set_normalization; predictions come back de-normalised with the
 * ensemble's spread.  X, T, mean and spread are DEVICE arrays.
 * mcml_mlp_predict runs every layer of every member in one launch when the
 * hidden width is a multiple of 64 and out_dim <= 3 (environment
 * MCML_MLP_FUSED=0: layer by layer, in chunks of `chunk` rows, 0 = 131072;
 * the two differ only in the order of the output layer's FP32 sums).
 */
typedef struct mcml_mlp_config {
  int32_t in_dim, hidden, depth, out_dim, ensemble;
  uint64_t seed;
  int32_t device;
  void *stream;
} mcml_mlp_config;
typedef struct mcml_mlp mcml_mlp;
int mcml_mlp_create(const mcml_mlp_config *cfg, mcml_mlp **mlp);
int mcml_mlp_set_normalization(mcml_mlp *mlp, const float *x_mean, const float *x_std,
                               const float *t_mean, const float *t_std);
int64_t mcml_mlp_num_params(const mcml_mlp *mlp);
/* FP32 parameters of one member (host), layer by layer: W (fan_in x
 * fan_out, row-major, fan_in of layer 0 padded to a multiple of 16) then b. */
int mcml_mlp_get_params(mcml_mlp *mlp, float *host, int member);
int mcml_mlp_set_params(mcml_mlp *mlp, const float *host, int member);
/* Loss and gradients of every member on rows [0, n) (no update; host out). */
int mcml_mlp_gradients(mcml_mlp *mlp, const float *X, const float *T, int n, float *loss,
                       float *grads);
int mcml_mlp_train_epoch(mcml_mlp *mlp, const float *X, const float *T, uint64_t n,
                         uint32_t batch, float lr, uint64_t shuffle_seed, float *loss);
int mcml_mlp_predict(mcml_mlp *mlp, const float *X, uint64_t n, float *mean, float *spread,
                     uint32_t chunk);
int mcml_mlp_sync(mcml_mlp *mlp);
void mcml_mlp_destroy(mcml_mlp *mlp);

/* ---- first pass without device allocation ----------------------------- */
/*
 * No counterpart in the reference (its host allocates with cudaMalloc on
 * every run, transport.cu:1037-1097).  For callers that cannot allocate
 * device memory when they want photons walked: real-time pipelines whose
 * device memory is fixed at start-up (cudaMalloc can block and synchronise
 * the device mid-run), or processes whose GPU memory another framework's
 * pool already owns.
 *
 * The walk's scratch memory is a fixed array of MCML_NOALLOC_SCRATCH_BYTES
 * inside the library, present on every GPU that loads it until the process
 * exits; it holds at most MCML_NOALLOC_MAX_SLOTS slot states, enough for the
 * reference's one-photon-per-thread layout on a B200 (303104).  The call
 * enqueues the first pass on `stream` (NULL = the legacy default stream)
 * and returns without waiting; *out (a DEVICE pointer the caller owns)
 * receives the per-SDS counts and FP64 weight sums when the stream reaches
 * it.  slots = 0 picks min(N, MCML_NOALLOC_MAX_SLOTS); larger values are
 * rejected with MCML_E_INVALID.  The same seed and slots give the same
 * counts as mcml_run.  No detection records are kept (use mcml_run for the
 * replay).  The first call on a device does its set-up (it looks up the
 * array's device address), and so does the first call after that device's
 * context was reset; make that first call before any stream capture.
 * All calls share the one array, which keeps the last call's contents;
 * each call clears what must start at zero, and calls that overlap on the
 * GPU (different streams or host threads) race -- serialise them.
 */
#define MCML_NOALLOC_SCRATCH_BYTES (8u << 20)
#define MCML_NOALLOC_MAX_SLOTS ((MCML_NOALLOC_SCRATCH_BYTES - 1024u) / 24u)
typedef struct mcml_noalloc_result {
  uint64_t detected[MCML_MAX_SDS];
  double weight_sum[MCML_MAX_SDS];
  double weight_sumsq[MCML_MAX_SDS];
  uint64_t steps;
} mcml_noalloc_result;
int mcml_run_noalloc(const mcml_sim *sim, uint64_t seed, uint64_t slots, int device,
                     void *stream, mcml_noalloc_result *out);

/* ---- checkpoint / resume of the first pass ----------------------------- */
/*
 * The first pass walked in launches of chunk_slots slots, with a
 * checkpoint file brought up to date after every launch -- the launch
 * boundary of the reference's host loop (transport.cu:114-150), where its
 * thread states, quotas and counters come back to the host.  Here a slot's
 * photons depend only on (seed, slot), so the checkpoint holds the slot
 * range done, the step count and the detection records so far; the slot
 * states are re-seeded.  If `path` exists, the run resumes after its last
 * completed launch; it must belong to the same simulation, seed,
 * slot_begin and slot count (else MCML_E_CHECKPOINT, the file untouched).
 * A resumed run detects the same photons as one uninterrupted mcml_run
 * with the same seed and slots; mcml_replay and the getters then work as
 * after mcml_run.  The file is append-only: records of a launch are
 * written and flushed before the header that counts them, so a crash
 * during an update leaves the previous checkpoint readable.
 *
 * File layout (little-endian): a 128-byte header {char magic[8]
 * "MCMLCKP1"; u32 version 1; u32 record_bytes 40; u64 run_digest, seed,
 * slot_begin, photons, slots, slots_done, records, steps, launches,
 * records_digest, header_digest; 24 zero bytes} followed by `records`
 * detection records {u64 photon; u32 sds; f32 weight; u32 xorwow d,
 * v[5]}.  Digests are 64-bit FNV-1a; header_digest covers the 96 bytes
 * before it, records_digest the record bytes in file order.
 */
typedef struct mcml_checkpoint_opts {
  const char *path;
  uint64_t chunk_slots; /* slots per launch; 0 = the larger of 32 slots per
                           resident thread and slots / 64                   */
  uint32_t max_chunks;  /* return MCML_INCOMPLETE after this many launches in
                           this call (0 = run to the end)                   */
  uint32_t reserved;
} mcml_checkpoint_opts;

typedef struct mcml_checkpoint_info {
  uint64_t seed, slot_begin, photons, slots;
  uint64_t slots_done, records, steps, launches;
} mcml_checkpoint_info;

/* MCML_OK when every slot is walked (result filled as by mcml_run),
 * MCML_INCOMPLETE when stopped by max_chunks (result untouched). */
int mcml_run_checkpointed(mcml_ctx *ctx, const mcml_checkpoint_opts *ck, mcml_result *result);
/* Reads and checks a checkpoint file on the host (no device needed). */
int mcml_checkpoint_read_info(const char *path, mcml_checkpoint_info *info);

/* ---- outputs from host data ------------------------------------------- */
/*
 * The same files as mcml_write_outputs, from host arrays instead of a
 * context: for results combined from several runs (replicas over
 * disjoint slot ranges on several GPUs, concatenated in slot order) or
 * kept from an earlier run.  Host only; no device is touched.
 */
typedef struct mcml_host_data {
  uint64_t photons;          /* the combined run's photon count (output scales)      */
  const uint64_t *detected;  /* num_sds detected counts                              */
  const double *weight_sum;  /* num_sds FP64 sums of detected weights (quanta)       */
  const float *const *rows;  /* num_sds pointers to detected[s] rows of L+2 floats,
                                photon order (pathlength_SDS_#); NULL without -R     */
  const uint64_t *A_rz;      /* num_sds x nz x nr u64 quanta, or NULL                */
  const uint64_t *A0_z;      /* num_sds x nz u64 quanta, or NULL                     */
  uint32_t grid_nr, grid_nz; /* 0 = the reference grid                               */
  float grid_dr, grid_dz;
  const char *gpu_name;      /* summary.json "sim_GPU"                               */
} mcml_host_data;
int mcml_write_host_outputs(const mcml_sim *sim, const mcml_host_data *data, const char *dir,
                            const char *output_txt, uint32_t flags, double sim_s,
                            double replay_s);

/* ---- text formatting ---------------------------------------------------- */
/*
 * The text pathlength_SDS_#.txt holds for n_rows rows of row_len floats
 * (io.cpp:313-323: every value in iostream's default format -- printf "%g",
 * 6 significant digits -- followed by a tab, each row by a newline).  The
 * text goes to out when it fits in capacity bytes; *written is its length
 * either way (out may be NULL to size it).  Host only.
 */
int mcml_format_rows_text(const float *rows, uint64_t n_rows, uint32_t row_len, char *out,
                          uint64_t capacity, uint64_t *written);

/* ---- test support ------------------------------------------------------ */
/*
 * The first count draws of curand_uniform on the XORWOW state
 * curand_init(seed, subsequence, 0) -- the stream the reference's thread
 * `subsequence` consumes (transport.cu:51-55, 733).  Host output buffer.
 * Used to feed recorded draws to the CPU oracle.
 */
int mcml_uniform_stream(int device, uint64_t seed, uint64_t subsequence,
                        uint64_t count, float *out);

/*
 * Known-answer probes of the walk's own device functions (spin,
 * transport.cu:742-786; Reflect, transport.cu:790-853), n samples, each
 * thread on its own XORWOW subsequence of `seed`.  out[2] (host):
 *   mcml_probe_spin:    mean cos(theta), mean cos^2(theta) of spin() with
 *                       anisotropy g applied to a photon going along +z;
 *   mcml_probe_reflect: fraction reflected at an interface n1 -> n2 for
 *                       incidence cosine cos_i, mean |dz| of the
 *                       transmitted photons.
 */
int mcml_probe_spin(int device, float g, uint64_t n, uint64_t seed, double *out);
int mcml_probe_reflect(int device, float n1, float n2, float cos_i, uint64_t n, uint64_t seed,
                       double *out);

#ifdef __cplusplus
}
#endif
#endif /* MCML_B200_H */
