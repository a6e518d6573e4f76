/*
 * empi_b200 -- C ABI of the B200 Matching Pursuit engine.
 *
 * Plain C types only: pointers, sizes, doubles.  Every call is synchronous
 * with respect to the caller's buffers (host data is copied before return);
 * device work runs on the engine's stream.  One engine per host thread, or
 * external locking.  Errors return an empi_status and leave a camelCase
 * message (the reference's exception texts where one exists) readable with
 * empi_last_error().
 *
 * Reference interfaces replaced (paths in the empi project):
 *   empi_workspace_*      Workspace / WorkspaceBuilder seam, inc/classes.hpp:63-80,
 *                         implemented there by GaborWorkspace (src/gabor.cpp:75-252)
 *   empi_subtract_atom_from_signal
 *                         Workspace::subtractAtomFromSignal, src/classes.cpp:15-22,
 *                         src/gabor.cpp:143-187
 *   empi_batch_*          Decomposition::compute and its SMP/MMP1/MMP2/MMP3
 *                         overrides (src/classes.cpp:26-87, src/mmp.cpp:9-45,
 *                         inc/mmp.hpp:11-31), run for many epochs at once
 *   empi_run_config       the empi CLI body, src/empi.cpp:49-167 (config file in,
 *                         SVAROG book out, stdout progress protocol)
 *   empi_book_write       BookWriter::write, src/io.cpp:104-168
 */
#ifndef EMPI_B200_H
#define EMPI_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EMPI_B200_ABI_VERSION 3

typedef enum {
    EMPI_OK = 0,
    EMPI_ERR_INVALID_ARGUMENT = 1,
    EMPI_ERR_CUDA = 2,
    EMPI_ERR_OUT_OF_MEMORY = 3,        /* insufficientMemory */
    EMPI_ERR_SIGNAL_IS_EMPTY = 4,      /* signalIsEmpty (src/classes.cpp:35-39) */
    EMPI_ERR_ENERGY_MAP_IS_EMPTY = 5,  /* energyMapIsEmpty (src/gabor.cpp:108-110) */
    EMPI_ERR_SIGNAL_TOO_LONG = 6,      /* signalFileIsTooLongForThisDecomposition */
    EMPI_ERR_CANDIDATE_OVERFLOW = 7,   /* candidates beyond the largest buffers the engine grows to */
    EMPI_ERR_CONFIG = 8,               /* configuration errors (src/empi.cpp:59-141) */
    EMPI_ERR_IO = 9,                   /* file errors (src/io.cpp) */
    EMPI_ERR_NO_DEVICE = 10,
    EMPI_ERR_INTERNAL = 11,
    EMPI_ERR_DEVICE_WAIT_TIMEOUT = 12  /* deviceWaitTimeout: a bounded device-side wait ran out */
} empi_status;

/* MP variants, src/empi.cpp:114-130 */
typedef enum { EMPI_SMP = 0, EMPI_MMP1 = 1, EMPI_MMP2 = 2, EMPI_MMP3 = 3 } empi_variant;

typedef struct empi_engine empi_engine;
typedef struct empi_workspace empi_workspace;
typedef struct empi_batch empi_batch;

/* Thread-local message of the last failed call ("" after success). */
const char* empi_last_error(void);
const char* empi_status_string(empi_status status);
int empi_abi_version(void);

/* ---------------------------------------------------------------- engine */

typedef struct {
    int device;              /* CUDA ordinal */
    void* stream;            /* cudaStream_t to run on; NULL = engine-owned stream */
    int transform_cap;       /* largest shared-memory sub-FFT (16..4096, power of 2); 0 = default */
    double candidate_band;   /* extra relative margin below the certified lower bound of the best
                                exact energy when selecting candidates (0 = none, the default:
                                the certified FP32 error bound alone decides) */
    int candidate_capacity;  /* initial candidate slots / bins per iteration over a batch
                                (0 = default); the buffers grow on demand */
    int iterations_per_graph;/* MP iterations per CUDA-graph launch; 0 = default */
    int timing;              /* nonzero: record CUDA events around every refresh launch */
    const char* tune_cache;  /* autotuner cache file (empi_b200/autotune.py) or NULL: batches
                                whose workload it holds take its tuned sub-FFT cap, iterations
                                per graph and per-size refresh variants (copied at creation) */
    int persistent;          /* run each chunk of MP iterations as one persistent cooperative
                                kernel instead of the multi-kernel CUDA graph: -1 = when the batch
                                is small (the default), 0 = never, 1 = whenever the batch allows it
                                (not with timing, a block proposal, the probe or pair collection) */
    int wait_limit_ms;       /* time limit of every device-side wait of the persistent kernel
                                (0 = default, 1000 ms); a wait that runs out ends the run with
                                EMPI_ERR_DEVICE_WAIT_TIMEOUT and leaves the context usable */
    int test_unreachable_wait; /* test hook, 0 in production: nonzero makes every grid barrier of
                                the persistent kernel wait for one block more than exist, so
                                the first wait runs out */
} empi_engine_opts;

void empi_engine_opts_default(empi_engine_opts* opts);
empi_status empi_engine_create(const empi_engine_opts* opts, empi_engine** out);
void empi_engine_destroy(empi_engine* engine);

/* GaborWorkspaceBuilder(energyError, scaleMin, scaleMax, freqMax), src/gabor.cpp:213 */
typedef struct {
    double energy_error;
    double scale_min;   /* seconds; 0 = default (2 samples) */
    double scale_max;   /* seconds; INFINITY = default (signal length) */
    double freq_max;    /* hertz; INFINITY = no limit */
} empi_dictionary;

/* Dictionary size (sum of fCount * tCount, GaborWorkspace::getAtomCount,
 * src/gabor.cpp:135-141) and scale count for a signal shape. */
empi_status empi_dictionary_size(const empi_dictionary* dict, double fs, int samples,
                                 uint64_t* atom_count, int* scale_count);

/* Scale table of a dictionary: s (seconds), Nfft, fCount, tCount per scale,
 * as the reference's prepareWorkspace builds them.  Arrays hold cap entries. */
empi_status empi_dictionary_scales(const empi_dictionary* dict, double fs, int samples, int cap,
                                   double* s, int* nfft, int* fcount, int* tcount, int* count);

/* Certified FP32 error bound of the engine's energy maps, per scale (no
 * counterpart in the reference, whose maps are FP64): for every bin of a
 * window whose channels' largest |sample| have norm B, the FP32 window value
 * is within bnd_d * B of the exact one, and
 *   (sqrt(e32 (1 - tau)) - d)^2 <= exact energy <= (sqrt(e32 (1 + tau)) + d)^2
 * with d = sqrt(Kc) bnd_d B, Kc = 2 sqrt(2) / (s fs), tau = (8 + 2 (C + 4)) 2^-24
 * for bins klo <= k <= khi, and d scaled by sqrt(rho), tau = tph + 2 (C + 4) 2^-24
 * for the phase-dependent bins k < klo or k > khi.  Candidates for the FP64
 * re-scoring are selected with these bounds, so the argmax is exact. */
empi_status empi_dictionary_error_bounds(const empi_dictionary* dict, double fs, int samples, int cap,
                                         float* bnd_d, float* rho, float* tph, int* klo, int* khi,
                                         int* count);

/* Tuned launch shape for a workload from an autotuner cache file, without a
 * GPU (no counterpart in the reference, which has no launch shapes): mode 0 =
 * single-channel MP loops (SMP, MMP2's channel sum), 1 = MMP1, 3 = MMP3;
 * channels per MP loop; samples 0 matches an entry tuned for uneven batches.
 * Returns EMPI_ERR_CONFIG ("noTunedEntry", "invalidTuneCache") when there is
 * none. */
empi_status empi_tune_lookup(const char* path, int mode, int channels, double fs, int samples,
                             double energy_error, int* transform_cap, int* iterations_per_graph,
                             int* wide_mask, int* persistent);

/* -------------------------------------------------- workspace (the seam) */

/* WorkspaceBuilder::prepareWorkspace(fs, channelCount, sampleCount, constraint),
 * inc/classes.hpp:76-80.  `variant` selects the constraint: EMPI_MMP1 applies
 * Mmp1Decomposition::constraint (src/mmp.cpp:9-21), the others none. */
empi_status empi_workspace_create(empi_engine* engine, const empi_dictionary* dict, double fs,
                                  int channels, int samples, empi_variant variant,
                                  empi_workspace** out);
void empi_workspace_destroy(empi_workspace* ws);

/* Workspace::compute(const MultiSignal&): samples are channel-major,
 * channels x samples doubles. */
empi_status empi_workspace_compute(empi_workspace* ws, const double* samples);

/* Workspace::findBestMatch(): writes channels x 6 params (modulus, amplitude,
 * t*fs, s*fs, f*2/fs, phase) as src/gabor.cpp:111-131; index (optional) gets
 * the winner's (scale, t, f) indices. */
empi_status empi_workspace_find_best(empi_workspace* ws, double* params, int* index);

/* Workspace::getAtomCount() */
empi_status empi_workspace_atom_count(const empi_workspace* ws, uint64_t* count);

/* Workspace::subtractAtom(atom, signal, channel): subtracts the atom from
 * `samples` (one channel, in/out, `samples` doubles long) and refreshes the
 * affected part of that channel's maps. */
empi_status empi_workspace_subtract_atom(empi_workspace* ws, const double* params,
                                         double* samples, int channel);

/* Energy maps of one scale for parity checks: energy [f][t] (fCount x tCount
 * floats, the FP32 values the engine ranks) -- optional, may be NULL. */
empi_status empi_workspace_energy_map(empi_workspace* ws, int scale, float* energy);

/* Workspace::subtractAtomFromSignal(atom, signal, fit): params (6, in/out when
 * fit), samples (in/out, n doubles). Runs on the engine's device. */
empi_status empi_subtract_atom_from_signal(empi_engine* engine, double* params, double* samples,
                                           int n, double fs, int fit);

/* Same as empi_subtract_atom_from_signal, for callers that cannot allocate
 * device memory: a host program whose device memory is owned by another
 * framework's pool allocator (a second allocator may find no memory left, and
 * cudaMalloc / cudaFree synchronise the whole device, stalling that
 * framework's streams), or a caller with a fixed device-memory budget that
 * rules out per-call allocations.  No counterpart in the reference: the
 * device copy of the signal and params lives in a fixed static device array
 * instead of per-call allocations, so n may not exceed
 * EMPI_NOALLOC_MAX_SAMPLES (8 MiB of doubles per device, held from library
 * load until exit; larger n fails with "signalLongerThanStaticScratch", n <= 0
 * with "invalidArgument").  `stream` is a cudaStream_t (NULL = the default
 * stream); the call waits for it before returning, and the caller's current
 * device is restored on every return.  The first call on a device looks up
 * the array's device address with that device current and caches it, so it
 * should come before any stream capture; a cudaDeviceReset of that device
 * afterwards is not supported (the cached address would be stale).  All
 * calls on a device share the array, so calls that overlap on the GPU (other
 * threads, other streams) race and must be serialised by the caller. */
#define EMPI_NOALLOC_MAX_SAMPLES (1 << 20)
empi_status empi_subtract_atom_from_signal_noalloc(int device, void* stream, double* params,
                                                   double* samples, int n, double fs, int fit);

/* ------------------------------------------------ batched decomposition */

/* DecompositionSettings, inc/classes.hpp:84-87 */
typedef struct {
    int iteration_max;
    double residual_energy;  /* stop when residue/total <= this; 1 - energyPercent/100 */
} empi_settings;

/* One epoch: samples x channels float32, sample-major (channels interleaved),
 * the layout of empi's input files (src/io.cpp:28-34). */
typedef struct {
    double fs;
    int channels;
    int samples;
    const float* data;
} empi_epoch;

/* Allocates device state for `count` epochs of the given shapes (data
 * pointers are not read).  All epochs use `variant`; each epoch's dictionary
 * follows its own fs and length. */
empi_status empi_batch_create(empi_engine* engine, empi_variant variant, const empi_dictionary* dict,
                              const empi_settings* settings, const empi_epoch* epochs, int count,
                              empi_batch** out);
void empi_batch_destroy(empi_batch* batch);

/* Copies each epoch's host data to the device (shapes must match). */
empi_status empi_batch_load(empi_batch* batch, const empi_epoch* epochs);

/* Runs the decomposition of all loaded epochs to completion. */
empi_status empi_batch_run(empi_batch* batch);

/* Atoms of one epoch: atoms[c][a][6] for c < channels, a < cap (same params
 * as find_best; MMP2 per-channel fits as src/mmp.cpp:36-43); count receives
 * the atom count per channel.  energies (optional): residual energy after
 * each iteration of the loop that produced the channel's atoms
 * ([channel][cap] for SMP, [cap] otherwise; NaN where none was computed).
 * indices (optional): (scale, t, f) per atom, same layout as energies x 3.
 * The first read after a run copies the whole batch's results to the host in
 * a few bulk copies; later reads of any epoch (this call and
 * empi_batch_total_energy) are served from that copy until the next load or
 * run. */
empi_status empi_batch_atoms(empi_batch* batch, int epoch, int cap, double* atoms, int* count,
                             double* energies, int* indices);

/* Total energy (src/classes.cpp:35, sum x^2 / fs) of each MP loop of an
 * epoch: one per channel for SMP, one otherwise (the channel sum for MMP2). */
empi_status empi_batch_total_energy(empi_batch* batch, int epoch, double* totals);

typedef struct {
    int iterations;           /* MP iterations run (max over loops) */
    int atoms;                /* atoms emitted over all loops */
    long long refresh_units;  /* shared-memory FFT work units executed */
    long long windows;        /* (window, group) slots recomputed */
    double fft_flops;         /* reference-equivalent FFT flops executed: 2.5 Nfft log2 Nfft per window */
    double algorithmic_bytes; /* compulsory HBM bytes of the refreshes: residual spans + slot writes */
    double refresh_ms;        /* summed CUDA-event time of refresh launches (timing opt) */
    int refresh_launches;
    int kernel_launches;      /* kernels launched by the last run */
    int candidate_bins;       /* FP64 re-scored bins over the last run */
    double run_ms;            /* device time of the last empi_batch_run */
    int transform_cap;        /* launch shape in use: largest sub-FFT, */
    int iterations_per_graph; /* MP iterations per graph launch, */
    int wide_mask;            /* sub-FFT sizes (bit log2 L) with one 128-register CTA per SM, */
    int tuned;                /* and whether it came from the tune cache */
    int sizes_mask;           /* sub-FFT sizes (bit log2 L) the batch's dictionaries use */
    /* proposal-ceiling probe (empi_batch_probe_proposal), summed over the run:
     * slots the refresh rule recomputed, and those of them whose upper bound,
     * propagated through the subtraction without recomputing, still reached
     * the next certified best value (no exact proposal could skip them), with
     * their reference-equivalent FFT work */
    long long probe_dirty_slots, probe_needed_slots;
    double probe_dirty_work, probe_needed_work;
    /* block proposal (empi_batch_set_proposal): iterations that used one, and
     * how many of their atoms lay in a proposed block (the hit rate) */
    int proposal_iterations, proposal_hits;
    int persistent;           /* 1: the run's MP iterations ran as the persistent kernel */
} empi_batch_stats;

empi_status empi_batch_get_stats(empi_batch* batch, empi_batch_stats* stats);

/* Enables (nonzero) or disables the proposal-ceiling probe of later runs (no
 * counterpart in the reference).  A block proposal can skip a window's
 * refresh only where a certified bound excludes it; the probe measures, on
 * the plain decomposition, the share of the refresh rule's work (reference
 * src/gabor.cpp:189-209) that no such proposal could skip.  Costs one float
 * per slot and two extra kernels per iteration; the atoms are unchanged. */
empi_status empi_batch_probe_proposal(empi_batch* batch, int enable);

/* Block proposal for later runs (no counterpart in the reference; it changes
 * how much of the refresh rule's work, src/gabor.cpp:189-209, is done, never
 * the atoms).  After each subtraction a proposer scores 16 scale bands x 32
 * time tiles; the dirty windows in the top k blocks are refreshed first, the
 * other dirty windows get certified upper bounds propagated through the
 * subtraction, and a second round refreshes those whose bound still reaches
 * the best certified lower bound.  source: 0 the learned network (weights:
 * a file written by empi_b200/proposal.py), 1 the blocks nearest the last
 * atom, 2 none (k ignored: only the certified second round), -1 off.  The
 * batch statistics report the hit rate.  Not for MMP1 (its constrained
 * energy is not a norm of the window values). */
empi_status empi_batch_set_proposal(empi_batch* batch, int source, int k, const char* weights);

/* Training data for the learned proposal (no counterpart in the reference):
 * with collection enabled, later runs keep the normalised 64 x 128
 * log-spectrogram of every MP loop's residual before each selection;
 * empi_batch_pairs then returns up to cap (spectrogram, block of the atom
 * that selection chose) pairs -- spec: cap x 8192 floats, block: cap ints
 * (band * 32 + tile) -- and their total in count. */
empi_status empi_batch_collect_pairs(empi_batch* batch, int enable);
empi_status empi_batch_pairs(empi_batch* batch, int cap, float* spec, int* block, int* count);

/* The device index of one MP loop (instance: 0 .. loops - 1 in batch order,
 * an SMP channel or an MMP epoch), the counterpart of inspecting the
 * reference's Heap (inc/heap.hpp:13-94): its slot keys (upper-bound float bits
 * << 32 | lower-bound float bits) and its tournament tree's leaf chunks
 * (chunks: upper bits << 32 | slot index of the chunk's maximum; chunk_l: the
 * chunk's largest lower bound).  Pass null arrays to get the sizes only. */
empi_status empi_batch_tree(empi_batch* batch, int instance, long long slot_cap, unsigned long long* slots,
                            long long* slot_count, int chunk_cap, unsigned long long* chunks, unsigned* chunk_l,
                            int* chunk_count);

/* The proposal network on a GPU, host arrays in and out (no counterpart in
 * the reference).  Weights: empi_proposal_parameter_count() floats in the
 * order of empi_b200/csrc/proposal.hpp.  scores: n x 512 block scores of n
 * spectrograms, with BF16 tensor cores (bf16 = 1) or in FP32.  gradients:
 * FP32 forward and backward of the mean softmax cross-entropy over n
 * (spectrogram, block) pairs.  train: SGD with momentum, `epochs` shuffled
 * passes in minibatches of `batch`, weights updated in place, each epoch's
 * mean loss in losses (optional). */
int empi_proposal_parameter_count(void);
empi_status empi_proposal_scores(int device, const float* spec, int n, const float* weights, int bf16,
                                 float* scores);
empi_status empi_proposal_gradients(int device, const float* spec, const int* labels, int n,
                                    const float* weights, float* grads, float* loss);
empi_status empi_proposal_train(int device, const float* spec, const int* labels, int n, int epochs, int batch,
                                float lr, float momentum, unsigned seed, float* weights, float* losses);

/* One-shot convenience: create + load + run; atoms of epoch e go to
 * atoms + e * channels_e * cap * 6 in order (counts likewise per channel). */
empi_status empi_decompose(empi_engine* engine, empi_variant variant, const empi_dictionary* dict,
                           const empi_settings* settings, const empi_epoch* epochs, int count,
                           int cap, double* atoms, int* counts);

/* ------------------------------------------------------ host surface */

/* Runs a complete empi job from a config file (src/empi.cpp:49-167):
 * reads the signal, decomposes on the GPU, writes the SVAROG book and
 * prints the START/CHANNEL/ATOM/END protocol to stdout. */
empi_status empi_run_config(const char* config_path, const empi_engine_opts* opts);

/* BookWriter::write for one epoch (src/io.cpp:104-168); `header` nonzero
 * writes the file header first (epoch 1).  samples: channels x n floats
 * channel-major; atoms: [c][cap][6]; counts per channel. */
empi_status empi_book_write(const char* path, int append, int epoch_number, double fs, int channels,
                            int n, const float* samples, int cap, const double* atoms,
                            const int* counts);

#ifdef __cplusplus
}
#endif

#endif /* EMPI_B200_H */
