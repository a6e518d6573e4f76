// Host engine: device state of batches and workspaces, CUDA-graph capture of
// the MP iteration, and the C ABI declared in include/empi_b200.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/empi_b200.h"
#include "engine.hpp"
#include "geometry.hpp"
#include "kernels.cuh"
#include "proposal.hpp"
#include "refresh_kernels.hpp"
#include "tune.hpp"

using namespace empi;

// ------------------------------------------------------------ errors

namespace {
thread_local std::string g_last_error;
}

namespace empi {

empi_status fail(empi_status st, const std::string& msg) {
    g_last_error = msg;
    return st;
}

empi_status ok() {
    g_last_error.clear();
    return EMPI_OK;
}

}  // namespace empi

#define CUDA_TRY(expr)                                                                     \
    do {                                                                                   \
        cudaError_t e_ = (expr);                                                           \
        if (e_ != cudaSuccess) {                                                           \
            return fail(e_ == cudaErrorMemoryAllocation ? EMPI_ERR_OUT_OF_MEMORY : EMPI_ERR_CUDA, \
                        e_ == cudaErrorMemoryAllocation ? std::string("insufficientMemory")  \
                                                        : std::string("cuda: ") + cudaGetErrorString(e_) + " (" #expr ")"); \
        }                                                                                  \
    } while (0)

extern "C" const char* empi_last_error(void) { return g_last_error.c_str(); }

extern "C" int empi_abi_version(void) { return EMPI_B200_ABI_VERSION; }

extern "C" const char* empi_status_string(empi_status st) {
    switch (st) {
        case EMPI_OK: return "ok";
        case EMPI_ERR_INVALID_ARGUMENT: return "invalidArgument";
        case EMPI_ERR_CUDA: return "cudaError";
        case EMPI_ERR_OUT_OF_MEMORY: return "insufficientMemory";
        case EMPI_ERR_SIGNAL_IS_EMPTY: return "signalIsEmpty";
        case EMPI_ERR_ENERGY_MAP_IS_EMPTY: return "energyMapIsEmpty";
        case EMPI_ERR_SIGNAL_TOO_LONG: return "signalFileIsTooLongForThisDecomposition";
        case EMPI_ERR_CANDIDATE_OVERFLOW: return "candidateOverflow";
        case EMPI_ERR_CONFIG: return "configurationError";
        case EMPI_ERR_IO: return "ioError";
        case EMPI_ERR_NO_DEVICE: return "noCudaDevice";
        case EMPI_ERR_INTERNAL: return "internalError";
        case EMPI_ERR_DEVICE_WAIT_TIMEOUT: return "deviceWaitTimeout";
    }
    return "unknown";
}

// ------------------------------------------------------------ engine

constexpr int kSizes = kRefreshSizes;  // sub-FFT sizes 2^0 .. 2^12, one refresh kernel each
// batches whose slot keys x channels per MP loop stay within this run the
// persistent kernel by default (measured on a B200: 0.70-0.89x of the graph's
// time at 4.6k-32k, equal at 69k, 1.1-1.45x slower from 75k on, where each
// per-instance step's own latency, not launch latency, bounds an iteration)
constexpr long long kPersistAutoWork = 1LL << 15;

struct empi_engine {
    empi_engine_opts opts;
    int device = 0;
    int sms = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    float2* tw = nullptr;
    cudaStream_t aux[kSizes] = {};     // branches of the per-size refresh fork
    cudaEvent_t fork = nullptr, join[kSizes] = {};
    RefreshKernels rk[3];              // SMP / MMP2 sum, MMP1, MMP3
    std::string tune_cache;            // autotuner cache file ("" = none)
};

extern "C" void empi_engine_opts_default(empi_engine_opts* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->transform_cap = 4096;
    o->candidate_band = 0.0;
    o->candidate_capacity = 0;
    o->iterations_per_graph = 8;
    o->persistent = -1;
    o->wait_limit_ms = 1000;
}

namespace {

empi_status set_device(const empi_engine* e) {
    CUDA_TRY(cudaSetDevice(e->device));
    return EMPI_OK;
}

}  // namespace

extern "C" empi_status empi_engine_create(const empi_engine_opts* opts, empi_engine** out) {
    if (!out) return fail(EMPI_ERR_INVALID_ARGUMENT, "invalidArgument");
    *out = nullptr;
    std::unique_ptr<empi_engine> e(new empi_engine);
    empi_engine_opts_default(&e->opts);
    if (opts) {
        e->opts = *opts;
        if (e->opts.transform_cap == 0) e->opts.transform_cap = 4096;
        if (!(e->opts.candidate_band >= 0.0) || e->opts.candidate_band >= 1.0) e->opts.candidate_band = 0.0;
        if (e->opts.iterations_per_graph <= 0) e->opts.iterations_per_graph = 8;
        if (e->opts.persistent < -1 || e->opts.persistent > 1) e->opts.persistent = -1;
        if (e->opts.wait_limit_ms <= 0) e->opts.wait_limit_ms = 1000;
    }
    int n = 0;
    cudaError_t ce = cudaGetDeviceCount(&n);
    if (ce != cudaSuccess || n == 0) return fail(EMPI_ERR_NO_DEVICE, "noCudaDevice");
    e->device = e->opts.device;
    if (e->device < 0 || e->device >= n) return fail(EMPI_ERR_INVALID_ARGUMENT, "invalidDevice");
    CUDA_TRY(cudaSetDevice(e->device));
    cudaDeviceProp prop;
    CUDA_TRY(cudaGetDeviceProperties(&prop, e->device));
    if (prop.major < 10) return fail(EMPI_ERR_NO_DEVICE, "deviceIsNotSm100");
    e->sms = prop.multiProcessorCount;
    if (e->opts.stream) {
        e->stream = (cudaStream_t)e->opts.stream;
    } else {
        CUDA_TRY(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
        e->own_stream = true;
    }
    // coarse table W_kTwN^m, then fine table W_(2^26)^m (twiddle_pow2)
    std::vector<float2> tw(2 * kTwN);
    for (int m = 0; m < kTwN; ++m) {
        const long double two_pi = 6.283185307179586476925286766559005768L;
        const long double a = two_pi * (long double)m / (long double)kTwN;
        const long double af = two_pi * (long double)m / (long double)(1ll << kTwFineLog);
        tw[m] = make_float2((float)cosl(a), (float)(-sinl(a)));
        tw[kTwN + m] = make_float2((float)cosl(af), (float)(-sinl(af)));
    }
    CUDA_TRY(cudaMalloc(&e->tw, sizeof(float2) * 2 * kTwN));
    CUDA_TRY(cudaMemcpy(e->tw, tw.data(), sizeof(float2) * 2 * kTwN, cudaMemcpyHostToDevice));
    refresh_kernels_single(e->rk[0]);
    refresh_kernels_mmp1(e->rk[1]);
    refresh_kernels_mmp3(e->rk[2]);
    persist_kernel_single(e->rk[0]);
    persist_kernel_mmp1(e->rk[1]);
    persist_kernel_mmp3(e->rk[2]);
    if (e->opts.tune_cache) e->tune_cache = e->opts.tune_cache;
    e->opts.tune_cache = nullptr;  // the engine keeps its own copy
    CUDA_TRY(cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming));
    for (int i = 0; i < kSizes; ++i) {
        CUDA_TRY(cudaStreamCreateWithFlags(&e->aux[i], cudaStreamNonBlocking));
        CUDA_TRY(cudaEventCreateWithFlags(&e->join[i], cudaEventDisableTiming));
    }
    *out = e.release();
    return ok();
}

extern "C" void empi_engine_destroy(empi_engine* e) {
    if (!e) return;
    cudaSetDevice(e->device);
    if (e->tw) cudaFree(e->tw);
    for (int i = 0; i < kSizes; ++i) {
        if (e->aux[i]) cudaStreamDestroy(e->aux[i]);
        if (e->join[i]) cudaEventDestroy(e->join[i]);
    }
    if (e->fork) cudaEventDestroy(e->fork);
    if (e->own_stream && e->stream) cudaStreamDestroy(e->stream);
    delete e;
}

// ------------------------------------------------------------ dictionary queries

extern "C" empi_status empi_dictionary_size(const empi_dictionary* d, double fs, int samples, uint64_t* count,
                                            int* scales) {
    if (!d) return fail(EMPI_ERR_INVALID_ARGUMENT, "invalidArgument");
    DictPlan dp;
    std::vector<ScalePlan> sp;
    std::vector<float> et;
    std::string err;
    if (!build_dictionary(fs, samples, d->energy_error, d->scale_min, d->scale_max, d->freq_max, 4096, dp, sp, et,
                          nullptr, nullptr, err))
        return fail(err == "signalFileIsTooLongForThisDecomposition" ? EMPI_ERR_SIGNAL_TOO_LONG
                                                                     : EMPI_ERR_INVALID_ARGUMENT,
                    err);
    if (count) *count = dp.values;
    if (scales) *scales = dp.nscales;
    return ok();
}

extern "C" empi_status empi_dictionary_scales(const empi_dictionary* d, double fs, int samples, int cap, double* s,
                                              int* nfft, int* fcount, int* tcount, int* count) {
    if (!d) return fail(EMPI_ERR_INVALID_ARGUMENT, "invalidArgument");
    DictPlan dp;
    std::vector<ScalePlan> sp;
    std::vector<float> et;
    std::string err;
    if (!build_dictionary(fs, samples, d->energy_error, d->scale_min, d->scale_max, d->freq_max, 4096, dp, sp, et,
                          nullptr, nullptr, err))
        return fail(EMPI_ERR_INVALID_ARGUMENT, err);
    for (int i = 0; i < dp.nscales && i < cap; ++i) {
        if (s) s[i] = sp[i].s;
        if (nfft) nfft[i] = sp[i].nfft;
        if (fcount) fcount[i] = sp[i].fcount;
        if (tcount) tcount[i] = sp[i].tcount;
    }
    if (count) *count = dp.nscales;
    return ok();
}

extern "C" empi_status empi_dictionary_error_bounds(const empi_dictionary* d, double fs, int samples, int cap,
                                                    float* bnd_d, float* rho, float* tph, int* klo, int* khi,
                                                    int* count) {
    if (!d) return fail(EMPI_ERR_INVALID_ARGUMENT, "invalidArgument");
    DictPlan dp;
    std::vector<ScalePlan> sp;
    std::vector<float> et;
    std::string err;
    if (!build_dictionary(fs, samples, d->energy_error, d->scale_min, d->scale_max, d->freq_max, 4096, dp, sp, et,
                          nullptr, nullptr, err))
        return fail(EMPI_ERR_INVALID_ARGUMENT, err);
    for (int i = 0; i < dp.nscales && i < cap; ++i) {
        if (bnd_d) bnd_d[i] = sp[i].bnd_d;
        if (rho) rho[i] = sp[i].bnd_rho;
        if (tph) tph[i] = sp[i].bnd_tph;
        if (klo) klo[i] = sp[i].klo;
        if (khi) khi[i] = sp[i].khi;
    }
    if (count) *count = dp.nscales;
    return ok();
}

extern "C" empi_status empi_tune_lookup(const char* path, int mode, int channels, double fs, int samples,
                                        double energy_error, int* transform_cap, int* iterations_per_graph,
                                        int* wide_mask, int* persistent) {
    if (!path) return fail(EMPI_ERR_INVALID_ARGUMENT, "invalidArgument");
    TuneParams tp;
    std::string err;
    if (!tune_lookup(path, TuneKey{mode, channels, fs, samples, energy_error}, tp, err))
        return fail(EMPI_ERR_CONFIG, err);
    if (transform_cap) *transform_cap = tp.transform_cap;
    if (iterations_per_graph) *iterations_per_graph = tp.iterations_per_graph;
    if (wide_mask) *wide_mask = tp.wide_mask;
    if (persistent) *persistent = tp.persistent;
    return ok();
}

// ------------------------------------------------------------ batch state

namespace {

template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
    cudaError_t alloc(size_t count) {
        n = std::max<size_t>(count, 1);
        return cudaMalloc(&p, sizeof(T) * n);
    }
    // drops the contents: for scratch that is rebuilt every iteration
    cudaError_t realloc_discard(size_t count) {
        if (p) cudaFree(p);
        p = nullptr;
        return alloc(count);
    }
};

}  // namespace

struct empi_batch {
    empi_engine* eng = nullptr;
    int variant = 0, mode = MODE_SINGLE;
    empi_settings settings{};
    std::vector<DictPlan> dicts;
    std::vector<ScalePlan> scales;
    std::vector<float> etab;
    std::vector<WinGeom> wgeom;
    std::vector<float> whf;
    std::vector<InstPlan> insts;
    std::vector<int2> blk_ic;
    std::vector<int2> fit_map;      // MMP2: (instance, input channel)
    std::vector<empi_epoch> epochs; // shapes
    std::vector<long long> epoch_in_off;
    std::vector<int> epoch_first_inst;
    std::vector<int> epoch_first_fit;
    int cmax = 1, nij = 0;
    long long total_in = 0;
    int max_n = 0;

    DevBuf<ScalePlan> d_scales;
    DevBuf<DictPlan> d_dicts;
    DevBuf<InstPlan> d_insts;
    DevBuf<int2> d_blk_ic, d_fit_map;
    DevBuf<float> d_input, d_input_spare, d_residual32, d_etab, d_whf, d_chan_xmax;
    cudaStream_t copy_stream = nullptr;  // staged loads of the next batch (batch_stage)
    cudaEvent_t staged_ev = nullptr;
    bool staged = false;
    // host copy of the last run's results (per-instance state, energies,
    // indices, atoms, MMP2 channel fits), filled by a few bulk copies on the
    // first read after a run (fetch_results) instead of several small copies
    // per epoch and channel; invalid from the next load or run on
    struct {
        bool valid = false;
        std::vector<InstState> st;
        std::vector<double> en, atoms, fit;
        std::vector<int4> ind;
    } hm;
    DevBuf<WinGeom> d_wgeom;
    DevBuf<double> d_residual, d_atoms, d_energies, d_chan_energy, d_fit_atoms, d_stats;
    DevBuf<InstState> d_state;
    DevBuf<unsigned long long> d_slots, d_chunks;
    DevBuf<unsigned> d_chunk_l;
    DevBuf<int2> d_dirty, d_crange;
    DevBuf<int> d_ij_units, d_ij_chunks, d_inst_units, d_inst_chunks, d_ctr, d_inst_bins;
    DevBuf<CandSlot> d_cslots;
    DevBuf<CandBin> d_cbins;
    DevBuf<double2> d_cbin_v;
    DevBuf<int4> d_indices;
    DevBuf<float> d_dump, d_prop, d_pscores;
    DevBuf<double> d_probe;
    DevBuf<int2> d_prange, d_qrange;
    DevBuf<unsigned char> d_stale, d_qmark, d_chunk_stale;
    int prop_source = -1;  // block proposal: 0 learned network, 1 last-atom heuristic, 2 none (k = 0)
    ProposalNet net;       // the learned proposer's device weights and activations
    DevBuf<float> d_pairs; // training-pair collection: [instance][iteration][64 x 128] spectrograms
    bool collect = false;
    DevBuf<int4> d_units;
    DevBuf<int> d_lmeta;  // loff[16], lcap[16], lcount[16], lhead[16]
    std::vector<int> sizes;  // sub-FFT sizes (log2) present in the batch
    void* refresh_fn[kSizes] = {};
    void* collect_fn = nullptr;

    BatchDev dev{};
    int refresh_grid_lg[kSizes] = {};
    int collect_grid = 0, tree_grid = 0, rescore_grid = 0;
    // launch shape: largest sub-FFT, MP iterations per graph, per-size
    // one-CTA-per-SM refresh variants, and whether the tune cache set them
    int lcap = 4096, K = 8, wide_mask = 0;
    bool tuned = false;
    // the persistent kernel (persist.cuh): the tune cache's choice (-1: none),
    // whether this batch runs it, its grid and its barrier
    int tuned_persistent = -1;
    bool persistent = false;
    int persist_grid = 0;
    DevBuf<GridSync> d_gsync;
    size_t refresh_smem = 0;             // the candidate kernel's (largest layout)
    size_t refresh_smem_lg[kSizes] = {};  // per sub-FFT size

    cudaGraphExec_t graph = nullptr;
    int graph_iters = 0;
    std::vector<cudaEvent_t> ev;  // timing pairs around refresh launches
    int ev_used = 0;
    cudaEvent_t run_start = nullptr, run_stop = nullptr;

    empi_batch_stats stats{};
    int launches_per_iter = 10;
    int regrows = 0;  // candidate-buffer growths (overflow recoveries) so far
    int total_chunks = 0;  // leaf chunks of all instances
    long long total_slots = 0;      // slot keys of all instances
    long long total_slot_work = 0;  // ... each times its MP loop's channels

    ~empi_batch() {
        if (graph) cudaGraphExecDestroy(graph);
        if (copy_stream) cudaStreamSynchronize(copy_stream), cudaStreamDestroy(copy_stream);
        if (staged_ev) cudaEventDestroy(staged_ev);
        for (auto e : ev) cudaEventDestroy(e);
        if (run_start) cudaEventDestroy(run_start);
        if (run_stop) cudaEventDestroy(run_stop);
    }
};

namespace {

const RefreshKernels& kernels_of(const empi_engine* e, int mode) {
    return mode == MODE_SINGLE ? e->rk[0] : (mode == MODE_MMP1 ? e->rk[1] : e->rk[2]);
}

// Per sub-FFT size present in the batch: the refresh kernel (two CTAs per SM,
// or the one-CTA 128-register variant where the tuned shape says so), its
// shared memory, L1 carveout and a grid of SMs x resident CTAs; the collect
// kernel runs any size, so it takes the largest layout.
empi_status configure(empi_batch* b) {
    const RefreshKernels& rk = kernels_of(b->eng, b->mode);
    for (int lg : b->sizes) {
        const int wide = (b->wide_mask >> lg) & 1;
        void* fn = rk.refresh[lg][wide];
        const size_t smem = rk.smem[lg];
        CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        {
            // as much L1 as the resident CTAs' shared memory leaves (percent of the maximum carveout)
            const size_t ctas = wide ? 1 : 2;
            const int pct = (int)std::min<size_t>(100, (ctas * (smem + 1024) * 100 + 228 * 1024 - 1) / (228 * 1024));
            CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, pct));
        }
        int o = 0;
        CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, fn, kUnitThreads, smem));
        if (o < 1) return fail(EMPI_ERR_INTERNAL, "refreshKernelDoesNotFit");
        b->refresh_fn[lg] = fn;
        b->refresh_smem_lg[lg] = smem;
        b->refresh_grid_lg[lg] = b->eng->sms * o;
    }
    b->collect_fn = rk.collect;
    CUDA_TRY(cudaFuncSetAttribute(b->collect_fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rk.collect_smem));
    b->refresh_smem = rk.collect_smem;
    b->collect_grid = b->eng->sms;
    // The persistent kernel: the engine's option, else the tune cache's
    // choice, else small batches only (below kPersistAutoSlots slot keys the
    // per-iteration work is a few microseconds per step and the graph is bound
    // by launch latency; above it the graph's two-CTAs-per-SM refresh is
    // faster).  It needs one co-resident 512-thread CTA per SM.
    int want = b->eng->opts.persistent;
    if (want < 0) want = b->tuned_persistent;
    if (want < 0) want = b->total_slot_work <= kPersistAutoWork ? 1 : 0;
    b->persistent = false;
    int coop = 0;
    CUDA_TRY(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, b->eng->device));
    if (want == 1 && coop && rk.persist) {
        // the largest refresh layout plus the phases' static shared memory
        // must fit one CTA (MMP1's per-bin channel sums at small L do not)
        cudaFuncAttributes fa{};
        int optin = 0;
        CUDA_TRY(cudaFuncGetAttributes(&fa, rk.persist));
        CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, b->eng->device));
        int o = 0;
        if (fa.sharedSizeBytes + rk.persist_smem <= (size_t)optin &&
            cudaFuncSetAttribute(rk.persist, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rk.persist_smem) ==
                cudaSuccess &&
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, rk.persist, kUnitThreads, rk.persist_smem) ==
                cudaSuccess &&
            o >= 1) {
            b->persistent = true;
            b->persist_grid = b->eng->sms;
            CUDA_TRY(b->d_gsync.alloc(1));
        }
        cudaGetLastError();  // a layout that does not fit is not an error: the graph runs
    }
    return EMPI_OK;
}

// the per-size refresh kernels as parallel branches: fork from s, join into s
void launch_refresh(empi_batch* b, cudaStream_t s) {
    empi_engine* e = b->eng;
    void* args[] = {&b->dev};
    if (b->sizes.size() == 1) {
        cudaLaunchKernel(b->refresh_fn[b->sizes[0]], dim3(b->refresh_grid_lg[b->sizes[0]]), dim3(kUnitThreads), args,
                         b->refresh_smem_lg[b->sizes[0]], s);
        return;
    }
    cudaEventRecord(e->fork, s);
    for (size_t i = 0; i < b->sizes.size(); ++i) {
        cudaStreamWaitEvent(e->aux[i], e->fork, 0);
        cudaLaunchKernel(b->refresh_fn[b->sizes[i]], dim3(b->refresh_grid_lg[b->sizes[i]]), dim3(kUnitThreads), args,
                         b->refresh_smem_lg[b->sizes[i]], e->aux[i]);
        cudaEventRecord(e->join[i], e->aux[i]);
    }
    for (size_t i = 0; i < b->sizes.size(); ++i) cudaStreamWaitEvent(s, e->join[i], 0);
}

void launch_collect(empi_batch* b, cudaStream_t s) {
    void* args[] = {&b->dev};
    cudaLaunchKernel(b->collect_fn, dim3(b->collect_grid), dim3(kUnitThreads), args, b->refresh_smem, s);
}

// schedule + refresh + tree + root (the map update after a subtraction, or
// the initial pass)
void launch_update(empi_batch* b, int sched_mode, int only_scale, double tA, double sA, cudaStream_t s,
                   cudaEvent_t e0, cudaEvent_t e1) {
    const int ninst = (int)b->insts.size();
    cudaMemsetAsync(b->dev.lcount, 0, sizeof(int) * 2 * 16, s);  // lcount and lhead
    k_sched_a<<<ninst, 128, 0, s>>>(b->dev, sched_mode, only_scale, tA, sA);
    k_sched_b<<<1, std::min(1024, 32 * ((ninst + 31) / 32)), 0, s>>>(b->dev);
    if (b->dev.prop && sched_mode == SCHED_ITERATE) k_propagate<<<b->tree_grid, 256, 0, s>>>(b->dev);
    if (e0) cudaEventRecord(e0, s);
    launch_refresh(b, s);
    if (e1) cudaEventRecord(e1, s);
    k_tree<<<b->tree_grid, 256, 0, s>>>(b->dev);
}

// candidates -> FP64 rescore -> atom
void launch_select(empi_batch* b, cudaStream_t s, bool probe = false) {
    const int ninst = (int)b->insts.size();
    k_cand_slots<<<ninst, 256, 0, s>>>(b->dev);
    if (probe && b->dev.prop) k_probe<<<b->tree_grid, 256, 0, s>>>(b->dev);
    launch_collect(b, s);
    k_rescore<<<b->rescore_grid, 512, 0, s>>>(b->dev);
    k_select<<<ninst, 128, 0, s>>>(b->dev);
}

void launch_net(empi_batch* b, cudaStream_t s) { net_run(b->net, b->dev, b->dev.pscores, s); }

empi_status net_load(empi_batch* b, const char* path) {
    std::vector<float> w(kNetParams);
    std::string err;
    if (!read_weights(path, w.data(), &err)) return fail(EMPI_ERR_IO, err);
    if (!net_init(b->net, w.data(), (int)b->insts.size(), &err)) return fail(EMPI_ERR_CUDA, err);
    return EMPI_OK;
}

// the two rounds of an iteration with a block proposal (kernels.cuh, "block
// proposal"): the proposer scores blocks from the residual, round 1 refreshes
// the dirty windows of the top ones, the other dirty slots get propagated
// bounds, round 2 refreshes those still reaching the root's lower bound
void launch_proposal_update(empi_batch* b, cudaStream_t s, cudaEvent_t e0, cudaEvent_t e1) {
    const int ninst = (int)b->insts.size();
    // without a proposer (source 2, k = 0) no block is proposed: the proposed
    // ranges stay empty and round 1 has no unit, so neither runs
    const bool round1 = b->prop_source != 2;
    if (b->prop_source == 1) k_scores_last_atom<<<ninst, 256, 0, s>>>(b->dev);
    else if (b->prop_source == 0) launch_net(b, s);
    if (round1) k_topk_ranges<<<ninst, 256, 0, s>>>(b->dev);
    cudaMemsetAsync(b->dev.lcount, 0, sizeof(int) * 2 * 16, s);
    k_sched_a<<<ninst, 128, 0, s>>>(b->dev, SCHED_ITERATE, -1, 0.0, 0.0);
    k_sched_b<<<1, std::min(1024, 32 * ((ninst + 31) / 32)), 0, s>>>(b->dev);
    if (e0) cudaEventRecord(e0, s);
    if (round1) launch_refresh(b, s);
    k_propagate_stale<<<b->tree_grid, 256, 0, s>>>(b->dev);
    k_tree<<<b->tree_grid, 256, 0, s>>>(b->dev);
    k_root<<<ninst, 256, 0, s>>>(b->dev);
    k_qualify<<<b->tree_grid, 256, 0, s>>>(b->dev, b->total_chunks);
    cudaMemsetAsync(b->dev.lcount, 0, sizeof(int) * 2 * 16, s);
    k_round2_sched<<<ninst, 512, 0, s>>>(b->dev);
    k_chunk_prefix<<<1, std::min(1024, 32 * ((ninst + 31) / 32)), 0, s>>>(b->dev);
    launch_refresh(b, s);
    if (e1) cudaEventRecord(e1, s);
    k_tree<<<b->tree_grid, 256, 0, s>>>(b->dev);
}

void launch_iteration(empi_batch* b, cudaStream_t s, cudaEvent_t e0, cudaEvent_t e1) {
    // training pairs: the residual's spectrogram before each selection
    if (b->collect) spectrogram(b->dev, b->d_pairs.p, s);
    launch_select(b, s, true);
    k_subtract<<<(int)b->blk_ic.size(), 1024, 0, s>>>(b->dev);
    if (b->dev.prange) launch_proposal_update(b, s, e0, e1);
    else launch_update(b, SCHED_ITERATE, -1, 0.0, 0.0, s, e0, e1);
}

empi_status build_batch(empi_engine* eng, int variant, const empi_dictionary* dict, const empi_settings* settings,
                        const empi_epoch* epochs, int count, int result_iters, empi_batch** out) {
    if (!eng || !dict || !epochs || count <= 0 || !out) return fail(EMPI_ERR_INVALID_ARGUMENT, "invalidArgument");
    if (settings && settings->iteration_max <= 0) return fail(EMPI_ERR_INVALID_ARGUMENT, "invalidMaximalNumberOfIterations");
    if (settings && (settings->residual_energy < 0 || settings->residual_energy >= 1.0))
        return fail(EMPI_ERR_INVALID_ARGUMENT, "invalidEnergyPercentValue");
    if (variant < EMPI_SMP || variant > EMPI_MMP3) return fail(EMPI_ERR_INVALID_ARGUMENT, "unsupportedDecompositionType");
    empi_status st = set_device(eng);
    if (st != EMPI_OK) return st;
    std::unique_ptr<empi_batch> b(new empi_batch);
    b->eng = eng;
    b->variant = variant;
    b->settings = settings ? *settings : empi_settings{result_iters, 0.0};
    const int iters = b->settings.iteration_max;
    // the launch shape: the engine's, or the tune cache's entry for this
    // workload (mode, channels per MP loop, fs, samples -- 0 when uneven --,
    // energyError)
    b->lcap = eng->opts.transform_cap;
    b->K = eng->opts.iterations_per_graph;
    if (!eng->tune_cache.empty()) {
        bool multi0 = false, even = true;
        int loopC = -1;
        for (int e = 0; e < count; ++e) {
            const bool m = (variant == EMPI_MMP1 || variant == EMPI_MMP3) && epochs[e].channels > 1;
            multi0 = multi0 || m;
            const int lc = m ? epochs[e].channels : 1;
            if (loopC >= 0 && lc != loopC) loopC = 0;
            else if (loopC < 0) loopC = lc;
            even = even && epochs[e].samples == epochs[0].samples && epochs[e].fs == epochs[0].fs;
        }
        TuneKey key{!multi0 ? MODE_SINGLE : (variant == EMPI_MMP1 ? MODE_MMP1 : MODE_MMP3), loopC, epochs[0].fs,
                    even ? epochs[0].samples : 0, dict->energy_error};
        TuneParams tp;
        std::string terr;
        if (tune_lookup(eng->tune_cache.c_str(), key, tp, terr)) {
            if (tp.transform_cap >= 16 && tp.transform_cap <= 4096 && !(tp.transform_cap & (tp.transform_cap - 1)))
                b->lcap = tp.transform_cap;
            if (tp.iterations_per_graph > 0 && tp.iterations_per_graph <= 64) b->K = tp.iterations_per_graph;
            b->wide_mask = tp.wide_mask & ((1 << kSizes) - 1);
            b->tuned_persistent = tp.persistent;
            b->tuned = true;
        } else if (terr != "noTunedEntry") {
            return fail(EMPI_ERR_CONFIG, terr);
        }
    }
    std::map<std::pair<double, int>, int> dict_of;
    bool multi = false;
    for (int e = 0; e < count; ++e) {
        const empi_epoch& ep = epochs[e];
        if (ep.channels <= 0 || ep.samples <= 0) return fail(EMPI_ERR_INVALID_ARGUMENT, "invalidEpochShape");
        auto key = std::make_pair(ep.fs, ep.samples);
        if (!dict_of.count(key)) {
            DictPlan dp;
            std::string err;
            if (!build_dictionary(ep.fs, ep.samples, dict->energy_error, dict->scale_min, dict->scale_max,
                                  dict->freq_max, b->lcap, dp, b->scales, b->etab, &b->wgeom,
                                  &b->whf, err))
                return fail(err == "signalFileIsTooLongForThisDecomposition" ? EMPI_ERR_SIGNAL_TOO_LONG
                                                                             : EMPI_ERR_INVALID_ARGUMENT,
                            err);
            dict_of[key] = (int)b->dicts.size();
            b->dicts.push_back(dp);
        }
        b->epochs.push_back(ep);
        b->epoch_in_off.push_back(b->total_in);
        b->total_in += (long long)ep.channels * ep.samples;
        b->max_n = std::max(b->max_n, ep.samples);
        if ((variant == EMPI_MMP1 || variant == EMPI_MMP3) && ep.channels > 1) multi = true;
    }
    b->mode = !multi ? MODE_SINGLE : (variant == EMPI_MMP1 ? MODE_MMP1 : MODE_MMP3);
    long long res_off = 0, slot_off = 0, chunk_off = 0, out_off = 0;
    int ij_off = 0, cen_off = 0;
    for (int e = 0; e < count; ++e) {
        const empi_epoch& ep = epochs[e];
        const int d = dict_of[std::make_pair(ep.fs, ep.samples)];
        const DictPlan& dp = b->dicts[d];
        b->epoch_first_inst.push_back((int)b->insts.size());
        b->epoch_first_fit.push_back((int)b->fit_map.size());
        auto add = [&](int C, int chan0) {
            InstPlan ip{};
            ip.dict = d;
            ip.C = C;
            ip.epoch = e;
            ip.chan0 = chan0;
            ip.ij_off = ij_off;
            ip.cen_off = cen_off;
            ip.res_off = res_off;
            ip.slot_off = slot_off;
            ip.chunk_off = chunk_off;
            ip.out_off = out_off;
            ip.in_off = b->epoch_in_off[e];
            ip.in_channels = ep.channels;
            const int inst = (int)b->insts.size();
            for (int c = 0; c < C; ++c) b->blk_ic.push_back(make_int2(inst, c));
            b->insts.push_back(ip);
            ij_off += dp.nscales;
            cen_off += C;
            res_off += (long long)C * dp.N;
            slot_off += dp.slots;
            b->total_slot_work += dp.slots * C;
            chunk_off += dp.chunks;
            out_off += (long long)iters * C * 6;
            b->cmax = std::max(b->cmax, C);
        };
        const bool smp = variant == EMPI_SMP || ep.channels == 1;  // src/empi.cpp:118
        if (smp) {
            for (int c = 0; c < ep.channels; ++c) add(1, c);
        } else if (variant == EMPI_MMP2) {
            add(1, -2);
            for (int c = 0; c < ep.channels; ++c) b->fit_map.push_back(make_int2((int)b->insts.size() - 1, c));
        } else {
            add(ep.channels, -1);
        }
    }
    b->nij = ij_off;
    const int ninst = (int)b->insts.size();
    // per sub-FFT size: the units of a full pass (the most a round can append)
    long long lcapl[16] = {0};
    for (const InstPlan& ip : b->insts) {
        const DictPlan& dp = b->dicts[ip.dict];
        for (int j = 0; j < dp.nscales; ++j) {
            const ScalePlan& sp = b->scales[dp.scale0 + j];
            for (int g = 0; g < sp.G; ++g) {
                const int B = g >= 2 ? sp.B2 : sp.B1;
                lcapl[sp.logL] += (sp.tcount + B - 1) / B;
            }
        }
    }
    int lmeta[64] = {0};
    long long lsum = 0;
    for (int l = 0; l < 16; ++l) {
        if (lcapl[l] > 0 && l < kSizes) b->sizes.push_back(l);
        lmeta[l] = (int)lsum;
        lmeta[16 + l] = (int)lcapl[l];
        lsum += lcapl[l];
    }
    // kernels per MP iteration: k_cand_slots, k_collect, k_rescore, k_select,
    // k_subtract, k_sched_a/b, one refresh per size, k_tree
    b->launches_per_iter = 8 + (int)b->sizes.size();
    if (lsum > (1LL << 31) - 1) return fail(EMPI_ERR_SIGNAL_TOO_LONG, "batchTooLarge");
    const int band_cap = eng->opts.candidate_capacity > 0 ? eng->opts.candidate_capacity
                                                          : std::max(8192, 64 * ninst);
    CUDA_TRY(b->d_scales.alloc(b->scales.size()));
    CUDA_TRY(b->d_dicts.alloc(b->dicts.size()));
    CUDA_TRY(b->d_insts.alloc(ninst));
    CUDA_TRY(b->d_blk_ic.alloc(b->blk_ic.size()));
    CUDA_TRY(b->d_fit_map.alloc(b->fit_map.size()));
    CUDA_TRY(b->d_input.alloc(b->total_in));
    CUDA_TRY(b->d_residual.alloc(res_off));
    CUDA_TRY(b->d_residual32.alloc(res_off));
    CUDA_TRY(b->d_etab.alloc(b->etab.size()));
    CUDA_TRY(b->d_wgeom.alloc(b->wgeom.size()));
    CUDA_TRY(b->d_whf.alloc(b->whf.size()));
    CUDA_TRY(b->d_atoms.alloc(out_off));
    CUDA_TRY(b->d_energies.alloc((size_t)ninst * iters));
    CUDA_TRY(b->d_chan_energy.alloc(cen_off));
    CUDA_TRY(b->d_chan_xmax.alloc(cen_off));
    CUDA_TRY(b->d_fit_atoms.alloc(b->fit_map.size() * (size_t)iters * 6));
    CUDA_TRY(b->d_stats.alloc(4));
    CUDA_TRY(b->d_state.alloc(ninst));
    CUDA_TRY(b->d_slots.alloc(slot_off));
    CUDA_TRY(b->d_chunks.alloc(chunk_off));
    b->total_chunks = (int)chunk_off;
    b->total_slots = slot_off;
    CUDA_TRY(b->d_chunk_l.alloc(chunk_off));
    CUDA_TRY(b->d_dirty.alloc(ij_off));
    CUDA_TRY(b->d_crange.alloc(ij_off));
    CUDA_TRY(b->d_ij_units.alloc(ij_off + ninst));
    CUDA_TRY(b->d_ij_chunks.alloc(ij_off + ninst));
    CUDA_TRY(b->d_inst_units.alloc(ninst + 1));
    CUDA_TRY(b->d_inst_chunks.alloc(ninst + 1));
    CUDA_TRY(b->d_ctr.alloc(CTR_COUNT));
    CUDA_TRY(b->d_cslots.alloc(band_cap));
    CUDA_TRY(b->d_cbins.alloc(band_cap));
    CUDA_TRY(b->d_cbin_v.alloc((size_t)band_cap * b->cmax));
    const int inst_bin_cap = 512;
    CUDA_TRY(b->d_inst_bins.alloc((size_t)ninst * inst_bin_cap));
    CUDA_TRY(b->d_indices.alloc((size_t)ninst * iters));
    CUDA_TRY(b->d_units.alloc((size_t)lsum));
    CUDA_TRY(b->d_lmeta.alloc(64));
    cudaStream_t s = eng->stream;
    CUDA_TRY(cudaMemcpyAsync(b->d_scales.p, b->scales.data(), sizeof(ScalePlan) * b->scales.size(),
                             cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaMemcpyAsync(b->d_dicts.p, b->dicts.data(), sizeof(DictPlan) * b->dicts.size(),
                             cudaMemcpyHostToDevice, s));
    if (!b->etab.empty())
        CUDA_TRY(cudaMemcpyAsync(b->d_etab.p, b->etab.data(), sizeof(float) * b->etab.size(), cudaMemcpyHostToDevice,
                                 s));
    CUDA_TRY(cudaMemcpyAsync(b->d_wgeom.p, b->wgeom.data(), sizeof(WinGeom) * b->wgeom.size(), cudaMemcpyHostToDevice,
                             s));
    CUDA_TRY(cudaMemcpyAsync(b->d_whf.p, b->whf.data(), sizeof(float) * b->whf.size(), cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaMemcpyAsync(b->d_insts.p, b->insts.data(), sizeof(InstPlan) * ninst, cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaMemcpyAsync(b->d_blk_ic.p, b->blk_ic.data(), sizeof(int2) * b->blk_ic.size(),
                             cudaMemcpyHostToDevice, s));
    if (!b->fit_map.empty())
        CUDA_TRY(cudaMemcpyAsync(b->d_fit_map.p, b->fit_map.data(), sizeof(int2) * b->fit_map.size(),
                                 cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaMemsetAsync(b->d_chunks.p, 0, sizeof(unsigned long long) * b->d_chunks.n, s));
    CUDA_TRY(cudaMemsetAsync(b->d_chunk_l.p, 0, sizeof(unsigned) * b->d_chunk_l.n, s));
    CUDA_TRY(cudaMemsetAsync(b->d_slots.p, 0, sizeof(unsigned long long) * b->d_slots.n, s));
    CUDA_TRY(cudaMemsetAsync(b->d_ctr.p, 0, sizeof(int) * CTR_COUNT, s));
    CUDA_TRY(cudaMemcpyAsync(b->d_lmeta.p, lmeta, sizeof(lmeta), cudaMemcpyHostToDevice, s));

    BatchDev& d = b->dev;
    d.scales = b->d_scales.p;
    d.dicts = b->d_dicts.p;
    d.insts = b->d_insts.p;
    d.blk_ic = b->d_blk_ic.p;
    d.tw = eng->tw;
    d.input = b->d_input.p;
    d.ninst = ninst;
    d.nblk_ic = (int)b->blk_ic.size();
    d.cmax = b->cmax;
    d.iter_max = iters;
    d.mode = b->mode;
    d.residual_energy = b->settings.residual_energy;
    d.band = (float)eng->opts.candidate_band;
    d.cslot_cap = band_cap;
    d.cbin_cap = band_cap;
    d.inst_bin_cap = inst_bin_cap;
    d.residual = b->d_residual.p;
    d.residual32 = b->d_residual32.p;
    d.etab = b->d_etab.p;
    d.wtab = reinterpret_cast<const int4*>(b->d_wgeom.p);
    d.whf = b->d_whf.p;
    d.units = b->d_units.p;
    d.loff = b->d_lmeta.p;
    d.lcap = b->d_lmeta.p + 16;
    d.lcount = b->d_lmeta.p + 32;
    d.lhead = b->d_lmeta.p + 48;
    d.state = b->d_state.p;
    d.slots = b->d_slots.p;
    d.chunks = b->d_chunks.p;
    d.chunk_l = b->d_chunk_l.p;
    d.dirty = b->d_dirty.p;
    d.ij_units = b->d_ij_units.p;
    d.ij_chunks = b->d_ij_chunks.p;
    d.ij_crange = b->d_crange.p;
    d.inst_units = b->d_inst_units.p;
    d.inst_chunks = b->d_inst_chunks.p;
    d.ctr = b->d_ctr.p;
    d.cslots = b->d_cslots.p;
    d.cbins = b->d_cbins.p;
    d.cbin_v = b->d_cbin_v.p;
    d.inst_bins = b->d_inst_bins.p;
    d.atoms = b->d_atoms.p;
    d.energies = b->d_energies.p;
    d.indices = b->d_indices.p;
    d.chan_energy = b->d_chan_energy.p;
    d.chan_xmax = b->d_chan_xmax.p;
    d.stats = b->d_stats.p;
    d.dump = nullptr;
    st = configure(b.get());
    if (st != EMPI_OK) return st;
    d.gsync = b->d_gsync.p;
    d.wait_ns = (long long)eng->opts.wait_limit_ms * 1000000LL;
    d.wait_extra = eng->opts.test_unreachable_wait ? 1 : 0;
    b->tree_grid = eng->sms * 8;
    b->rescore_grid = eng->sms;
    if (b->max_n * sizeof(double) > 48 * 1024 && !b->fit_map.empty()) {
        CUDA_TRY(cudaFuncSetAttribute(k_mmp2_fit, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(b->max_n * sizeof(double))));
    }
    if (b->max_n * sizeof(double) > 200 * 1024 && !b->fit_map.empty())
        return fail(EMPI_ERR_INVALID_ARGUMENT, "epochTooLongForMmp2Fit");
    CUDA_TRY(cudaEventCreate(&b->run_start));
    CUDA_TRY(cudaEventCreate(&b->run_stop));
    CUDA_TRY(cudaStreamSynchronize(s));
    *out = b.release();
    return ok();
}

empi_status check_errors(empi_batch* b) {
    int chk = 0;
    CUDA_TRY(cudaMemcpyAsync(&chk, b->d_ctr.p + CTR_CHECK, sizeof(int), cudaMemcpyDeviceToHost, b->eng->stream));
    std::vector<InstState> st(b->insts.size());
    CUDA_TRY(cudaMemcpyAsync(st.data(), b->d_state.p, sizeof(InstState) * st.size(), cudaMemcpyDeviceToHost,
                             b->eng->stream));
    CUDA_TRY(cudaStreamSynchronize(b->eng->stream));
    if (chk) return fail(EMPI_ERR_INTERNAL, "boundsCheck:" + std::to_string(chk));  // EMPI_CHECK builds only
    for (size_t i = 0; i < st.size(); ++i) {
        if (st[i].status == ST_ERROR || st[i].err != ERR_NONE) {
            switch (st[i].err) {
                case ERR_SIGNAL_EMPTY: return fail(EMPI_ERR_SIGNAL_IS_EMPTY, "signalIsEmpty");
                case ERR_MAP_EMPTY: return fail(EMPI_ERR_ENERGY_MAP_IS_EMPTY, "energyMapIsEmpty");
                case ERR_CAND_OVERFLOW: return fail(EMPI_ERR_CANDIDATE_OVERFLOW, "candidateOverflow");
                default: return fail(EMPI_ERR_INTERNAL, "internalError");
            }
        }
    }
    return EMPI_OK;
}

// Grows the candidate buffers fourfold after an overflow stalled some
// instances (their contents are per-iteration scratch); the graph, which
// holds the old pointers, is captured again on the next run step.
empi_status grow_candidates(empi_batch* b) {
    BatchDev& d = b->dev;
    const long long cap = 4LL * std::max(d.cslot_cap, d.cbin_cap);
    const long long icap = 4LL * d.inst_bin_cap;
    // at most 2^24 candidate slots / bins (~0.8 GB with their FP64 values at
    // one channel) and 2^28 per-instance bin ids
    if (cap > (1LL << 24) || cap * b->cmax > (1LL << 26) || icap * (long long)b->insts.size() > (1LL << 28))
        return fail(EMPI_ERR_CANDIDATE_OVERFLOW, "candidateOverflow");
    CUDA_TRY(cudaStreamSynchronize(b->eng->stream));
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    CUDA_TRY(b->d_cslots.realloc_discard((size_t)cap));
    CUDA_TRY(b->d_cbins.realloc_discard((size_t)cap));
    CUDA_TRY(b->d_cbin_v.realloc_discard((size_t)cap * b->cmax));
    CUDA_TRY(b->d_inst_bins.realloc_discard((size_t)icap * b->insts.size()));
    d.cslots = b->d_cslots.p;
    d.cbins = b->d_cbins.p;
    d.cbin_v = b->d_cbin_v.p;
    d.inst_bins = b->d_inst_bins.p;
    d.cslot_cap = (int)cap;
    d.cbin_cap = (int)cap;
    d.inst_bin_cap = (int)icap;
    b->regrows++;
    return EMPI_OK;
}

// The persistent kernel runs when the batch chose it and nothing needs the
// multi-kernel form: per-kernel timing events, the block proposal, the probe
// or the training-pair collection.
bool runs_persistent(const empi_batch* b) {
    return b->persistent && !b->eng->opts.timing && !b->dev.prop && !b->dev.prange && !b->collect;
}

empi_status capture_graph(empi_batch* b) {
    const int K = b->K;
    const bool timing = b->eng->opts.timing != 0;
    if (timing && b->ev.empty()) {
        b->ev.resize(2 * (K + 1));
        for (auto& e : b->ev) CUDA_TRY(cudaEventCreate(&e));
    }
    if (b->graph || timing) return EMPI_OK;  // timing mode launches eagerly, events between kernels
    if (runs_persistent(b)) return EMPI_OK;
    cudaStream_t s = b->eng->stream;
    cudaGraph_t g = nullptr;
    CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < K; ++k) launch_iteration(b, s, nullptr, nullptr);
    cudaError_t ce = cudaStreamEndCapture(s, &g);
    if (ce != cudaSuccess) return fail(EMPI_ERR_CUDA, std::string("cuda: ") + cudaGetErrorString(ce));
    ce = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (ce != cudaSuccess) return fail(EMPI_ERR_CUDA, std::string("cuda: ") + cudaGetErrorString(ce));
    b->graph_iters = K;
    return EMPI_OK;
}

}  // namespace

extern "C" empi_status empi_batch_create(empi_engine* eng, empi_variant variant, const empi_dictionary* dict,
                                         const empi_settings* settings, const empi_epoch* epochs, int count,
                                         empi_batch** out) {
    if (!settings) return fail(EMPI_ERR_INVALID_ARGUMENT, "invalidArgument");
    return build_batch(eng, (int)variant, dict, settings, epochs, count, settings->iteration_max, out);
}

extern "C" void empi_batch_destroy(empi_batch* b) {
    if (!b) return;
    cudaSetDevice(b->eng->device);
    cudaStreamSynchronize(b->eng->stream);
    delete b;
}

extern "C" empi_status empi_batch_load(empi_batch* b, const empi_epoch* epochs) {
    if (!b || !epochs) return fail(EMPI_ERR_INVALID_ARGUMENT, "invalidArgument");
    empi_status st = set_device(b->eng);
    if (st != EMPI_OK) return st;
    for (size_t e = 0; e < b->epochs.size(); ++e) {
        if (epochs[e].channels != b->epochs[e].channels || epochs[e].samples != b->epochs[e].samples || !epochs[e].data)
            return fail(EMPI_ERR_INVALID_ARGUMENT, "epochShapeMismatch");
        CUDA_TRY(cudaMemcpyAsync(b->d_input.p + b->epoch_in_off[e], epochs[e].data,
                                 sizeof(float) * (size_t)epochs[e].channels * epochs[e].samples,
                                 cudaMemcpyHostToDevice, b->eng->stream));
    }
    CUDA_TRY(cudaStreamSynchronize(b->eng->stream));
    b->staged = false;  // these epochs replace any staged ones
    b->hm.valid = false;
    return ok();
}

namespace empi {

empi_status batch_load_device(empi_batch* b, const float* const* device_data) {
    b->hm.valid = false;
    for (size_t e = 0; e < b->epochs.size(); ++e)
        CUDA_TRY(cudaMemcpyAsync(b->d_input.p + b->epoch_in_off[e], device_data[e],
                                 sizeof(float) * (size_t)b->epochs[e].channels * b->epochs[e].samples,
                                 cudaMemcpyDeviceToDevice, b->eng->stream));
    return EMPI_OK;
}

}  // namespace empi

extern "C" empi_status empi_batch_run(empi_batch* b) { return batch_run_hooked(b, nullptr); }

namespace empi {

empi_status batch_stage(empi_batch* b, const empi_epoch* epochs) {
    if (!b || !epochs) return fail(EMPI_ERR_INVALID_ARGUMENT, "invalidArgument");
    empi_status st = set_device(b->eng);
    if (st != EMPI_OK) return st;
    if (!b->copy_stream) {
        CUDA_TRY(cudaStreamCreateWithFlags(&b->copy_stream, cudaStreamNonBlocking));
        CUDA_TRY(cudaEventCreateWithFlags(&b->staged_ev, cudaEventDisableTiming));
    }
    if (!b->d_input_spare.p) CUDA_TRY(b->d_input_spare.alloc(b->d_input.n));
    for (size_t e = 0; e < b->epochs.size(); ++e) {
        if (epochs[e].channels != b->epochs[e].channels || epochs[e].samples != b->epochs[e].samples || !epochs[e].data)
            return fail(EMPI_ERR_INVALID_ARGUMENT, "epochShapeMismatch");
        CUDA_TRY(cudaMemcpyAsync(b->d_input_spare.p + b->epoch_in_off[e], epochs[e].data,
                                 sizeof(float) * (size_t)epochs[e].channels * epochs[e].samples,
                                 cudaMemcpyHostToDevice, b->copy_stream));
    }
    CUDA_TRY(cudaEventRecord(b->staged_ev, b->copy_stream));
    b->staged = true;
    return ok();
}

empi_status batch_loop_progress(empi_batch* b, int epoch, int loop, int* it, int* running, double* etotal,
                                double* energies) {
    if (!b || epoch < 0 || epoch >= (int)b->epochs.size()) return fail(EMPI_ERR_INVALID_ARGUMENT, "invalidArgument");
    const int i0 = b->epoch_first_inst[epoch];
    const int loops = b->insts[i0].chan0 >= 0 ? b->epochs[epoch].channels : 1;
    if (loop < 0 || loop >= loops) return fail(EMPI_ERR_INVALID_ARGUMENT, "invalidArgument");
    const int inst = i0 + loop;
    InstState is;
    CUDA_TRY(cudaMemcpy(&is, b->d_state.p + inst, sizeof(is), cudaMemcpyDeviceToHost));
    *it = is.it;
    *running = is.status == ST_RUNNING || is.status == ST_STALLED;
    *etotal = is.etotal;
    if (energies && is.it > 0)
        CUDA_TRY(cudaMemcpy(energies, b->d_energies.p + (size_t)inst * b->settings.iteration_max,
                            sizeof(double) * is.it, cudaMemcpyDeviceToHost));
    return EMPI_OK;
}

empi_status batch_run_hooked(empi_batch* b, const std::function<void()>& after_chunk) {
    if (!b) return fail(EMPI_ERR_INVALID_ARGUMENT, "invalidArgument");
    empi_status st = set_device(b->eng);
    if (st != EMPI_OK) return st;
    b->hm.valid = false;
    st = capture_graph(b);
    if (st != EMPI_OK) return st;
    cudaStream_t s = b->eng->stream;
    if (b->staged) {
        // decompose the epochs staged by batch_stage: wait for their copy and
        // make their buffer the input (k_init and the MMP2 fit read it)
        CUDA_TRY(cudaStreamWaitEvent(s, b->staged_ev, 0));
        std::swap(b->d_input.p, b->d_input_spare.p);
        b->dev.input = b->d_input.p;
        b->staged = false;
    }
    const bool timing = b->eng->opts.timing != 0;
    CUDA_TRY(cudaMemsetAsync(b->d_ctr.p, 0, sizeof(int) * CTR_COUNT, s));
    CUDA_TRY(cudaMemsetAsync(b->d_stats.p, 0, sizeof(double) * 4, s));
    if (b->dev.probe) CUDA_TRY(cudaMemsetAsync(b->dev.probe, 0, sizeof(double) * 4, s));
    if (b->dev.qmark) CUDA_TRY(cudaMemsetAsync(b->dev.qmark, 0, b->d_qmark.n, s));
    CUDA_TRY(cudaMemsetAsync(b->d_energies.p, 0xff, sizeof(double) * b->d_energies.n, s));  // NaN
    CUDA_TRY(cudaEventRecord(b->run_start, s));
    k_init<<<(int)b->blk_ic.size(), 256, 0, s>>>(b->dev, 1);
    launch_update(b, SCHED_INIT, -1, 0.0, 0.0, s, timing ? b->ev[0] : nullptr, timing ? b->ev[1] : nullptr);
    int launches = 4 + (int)b->sizes.size();  // k_init, k_sched_a/b, refreshes, k_tree
    double refresh_ms = 0.0;
    int refresh_launches = 0;
    if (timing) {
        CUDA_TRY(cudaStreamSynchronize(s));
        float ms = 0.f;
        CUDA_TRY(cudaEventElapsedTime(&ms, b->ev[0], b->ev[1]));
        refresh_ms += ms;
        refresh_launches++;
    }
    const int imax = b->settings.iteration_max;
    const int K = b->K;
    const bool persistent = runs_persistent(b);
    // every instance stops itself after imax atoms; a chunk in which some
    // instances stall on a candidate overflow costs at most one extra chunk
    const int max_regrows = 12;
    const int max_chunks = (imax + K - 1) / K + max_regrows + 2;
    int chunks = 0;
    for (;;) {
        if (timing) {
            for (int k = 0; k < K; ++k) launch_iteration(b, s, b->ev[2 * (k + 1)], b->ev[2 * (k + 1) + 1]);
            CUDA_TRY(cudaGetLastError());
            launches += K * b->launches_per_iter;
        } else if (persistent) {
            // one cooperative launch per chunk: every CTA co-resident, or the
            // launch fails (no barrier can wait on a CTA that never runs)
            CUDA_TRY(cudaMemsetAsync(b->d_gsync.p, 0, sizeof(GridSync), s));
            int iters = K;
            void* args[] = {&b->dev, &iters};
            const RefreshKernels& rk = kernels_of(b->eng, b->mode);
            CUDA_TRY(cudaLaunchCooperativeKernel(rk.persist, dim3(b->persist_grid), dim3(kUnitThreads), args,
                                                 rk.persist_smem, s));
            launches += 1;
        } else {
            CUDA_TRY(cudaGraphLaunch(b->graph, s));
            launches += K * b->launches_per_iter;
        }
        ++chunks;
        int ctr_now[CTR_COUNT];
        GridSync gs{};
        CUDA_TRY(cudaMemcpyAsync(ctr_now, b->d_ctr.p, sizeof(ctr_now), cudaMemcpyDeviceToHost, s));
        if (persistent) CUDA_TRY(cudaMemcpyAsync(&gs, b->d_gsync.p, sizeof(gs), cudaMemcpyDeviceToHost, s));
        CUDA_TRY(cudaStreamSynchronize(s));
        if (gs.err) return fail(EMPI_ERR_DEVICE_WAIT_TIMEOUT, "deviceWaitTimeout:phase" + std::to_string(gs.err - 1));
        if (timing) {
            for (int k = 0; k < K; ++k) {
                float ms = 0.f;
                CUDA_TRY(cudaEventElapsedTime(&ms, b->ev[2 * (k + 1)], b->ev[2 * (k + 1) + 1]));
                refresh_ms += ms;
                refresh_launches++;
            }
        }
        if (after_chunk) after_chunk();
        if (ctr_now[CTR_STALLED] > 0) {
            // more candidates than the buffers hold: grow them, resume the
            // stalled instances (nothing of theirs moved in the stalled step)
            if (b->regrows >= max_regrows) return fail(EMPI_ERR_CANDIDATE_OVERFLOW, "candidateOverflow");
            st = grow_candidates(b);
            if (st != EMPI_OK) return st;
            st = capture_graph(b);
            if (st != EMPI_OK) return st;
            k_unstall<<<std::max(1, std::min(1024, ((int)b->insts.size() + 255) / 256)), 256, 0, s>>>(b->dev);
            CUDA_TRY(cudaGetLastError());
            ++launches;
        } else if (ctr_now[CTR_ACTIVE] == 0) {
            break;
        }
        if (chunks >= max_chunks) return fail(EMPI_ERR_INTERNAL, "iterationLimitExceeded");
    }
    if (!b->fit_map.empty()) {
        k_mmp2_fit<<<(int)b->fit_map.size(), 256, b->max_n * sizeof(double), s>>>(b->dev, b->d_fit_map.p,
                                                                                 b->d_fit_atoms.p, imax);
        launches++;
    }
    CUDA_TRY(cudaEventRecord(b->run_stop, s));
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(s));
    float run_ms = 0.f;
    CUDA_TRY(cudaEventElapsedTime(&run_ms, b->run_start, b->run_stop));
    int ctr[CTR_COUNT];
    double stats[4];
    CUDA_TRY(cudaMemcpy(ctr, b->d_ctr.p, sizeof(ctr), cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(stats, b->d_stats.p, sizeof(stats), cudaMemcpyDeviceToHost));
    std::vector<InstState> sts(b->insts.size());
    CUDA_TRY(cudaMemcpy(sts.data(), b->d_state.p, sizeof(InstState) * sts.size(), cudaMemcpyDeviceToHost));
    b->stats = empi_batch_stats{};
    int maxit = 0, natoms = 0;
    for (auto& x : sts) {
        maxit = std::max(maxit, x.it);
        natoms += x.it;
    }
    b->stats.iterations = maxit;
    b->stats.atoms = natoms;
    b->stats.refresh_units = ctr[CTR_STAT_UNITS];
    b->stats.windows = (long long)stats[2];
    b->stats.fft_flops = stats[0];
    b->stats.refresh_ms = refresh_ms;
    b->stats.refresh_launches = refresh_launches;
    b->stats.kernel_launches = launches;
    b->stats.candidate_bins = ctr[CTR_STAT_BINS];
    b->stats.run_ms = run_ms;
    b->stats.algorithmic_bytes = stats[1];
    b->stats.transform_cap = b->lcap;
    b->stats.iterations_per_graph = b->K;
    b->stats.wide_mask = b->wide_mask;
    b->stats.tuned = b->tuned ? 1 : 0;
    b->stats.proposal_iterations = ctr[CTR_PROP_ITERS];
    b->stats.proposal_hits = ctr[CTR_PROP_HITS];
    b->stats.persistent = persistent ? 1 : 0;
    if (b->dev.probe) {
        double pr[4];
        CUDA_TRY(cudaMemcpy(pr, b->dev.probe, sizeof(pr), cudaMemcpyDeviceToHost));
        b->stats.probe_dirty_slots = (long long)pr[0];
        b->stats.probe_needed_slots = (long long)pr[1];
        b->stats.probe_dirty_work = pr[2];
        b->stats.probe_needed_work = pr[3];
    }
    for (int lg : b->sizes) b->stats.sizes_mask |= 1 << lg;
    empi_status es = check_errors(b);
    if (es != EMPI_OK) return es;
    return ok();
}

}  // namespace empi

extern "C" empi_status empi_batch_set_proposal(empi_batch* b, int source, int k, const char* weights) {
    if (!b || source < -1 || source > 2 || k < 0 || k > kProposalBlocks || (source == 0 && !weights))
        return fail(EMPI_ERR_INVALID_ARGUMENT, "invalidArgument");
    if (source >= 0 && b->mode == MODE_MMP1) return fail(EMPI_ERR_INVALID_ARGUMENT, "proposalUnsupportedForMmp1");
    if (source >= 0 && b->dev.prop) return fail(EMPI_ERR_INVALID_ARGUMENT, "proposalWithProbe");
    empi_status st = set_device(b->eng);
    if (st != EMPI_OK) return st;
    CUDA_TRY(cudaStreamSynchronize(b->eng->stream));
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    b->prop_source = source;
    if (source < 0) {
        b->dev.pscores = nullptr;
        b->dev.prange = nullptr;
        b->dev.qrange = nullptr;
        b->dev.stale = nullptr;
        b->dev.qmark = nullptr;
        b->dev.chunk_stale = nullptr;
        return ok();
    }
    if (source == 0) {
        st = net_load(b, weights);
        if (st != EMPI_OK) return st;
    }
    const size_t nij = b->nij;
    if (!b->d_pscores.p) CUDA_TRY(b->d_pscores.alloc(b->insts.size() * (size_t)kProposalBlocks));
    if (!b->d_prange.p) CUDA_TRY(b->d_prange.alloc(nij));
    if (!b->d_qrange.p) CUDA_TRY(b->d_qrange.alloc(nij));
    std::vector<int2> empty(nij, make_int2(0, -1)), qinit(nij, make_int2(0x7fffffff, -1));
    CUDA_TRY(cudaMemcpy(b->d_prange.p, empty.data(), sizeof(int2) * nij, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(b->d_qrange.p, qinit.data(), sizeof(int2) * nij, cudaMemcpyHostToDevice));
    b->dev.pscores = b->d_pscores.p;
    b->dev.prange = b->d_prange.p;
    b->dev.qrange = b->d_qrange.p;
    b->dev.prop_k = source == 2 ? 0 : k;
    if (!b->d_stale.p) CUDA_TRY(b->d_stale.alloc(b->d_slots.n));
    CUDA_TRY(cudaMemset(b->d_stale.p, 0, b->d_stale.n));
    b->dev.stale = b->d_stale.p;
    if (!b->d_qmark.p) CUDA_TRY(b->d_qmark.alloc(b->d_slots.n));
    CUDA_TRY(cudaMemset(b->d_qmark.p, 0, b->d_qmark.n));
    b->dev.qmark = b->d_qmark.p;
    if (!b->d_chunk_stale.p) CUDA_TRY(b->d_chunk_stale.alloc(b->d_chunks.n));
    CUDA_TRY(cudaMemset(b->d_chunk_stale.p, 0, b->d_chunk_stale.n));
    b->dev.chunk_stale = b->d_chunk_stale.p;
    return ok();
}

extern "C" empi_status empi_batch_collect_pairs(empi_batch* b, int enable) {
    if (!b) return fail(EMPI_ERR_INVALID_ARGUMENT, "invalidArgument");
    empi_status st = set_device(b->eng);
    if (st != EMPI_OK) return st;
    CUDA_TRY(cudaStreamSynchronize(b->eng->stream));
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    if (enable && !b->d_pairs.p)
        CUDA_TRY(b->d_pairs.alloc(b->insts.size() * (size_t)b->settings.iteration_max * kSpecSize));
    b->collect = enable != 0;
    return ok();
}

extern "C" empi_status empi_batch_pairs(empi_batch* b, int cap, float* spec, int* block, int* count) {
    if (!b || !count || cap < 0 || (cap > 0 && (!spec || !block))) return fail(EMPI_ERR_INVALID_ARGUMENT, "invalidArgument");
    if (!b->d_pairs.p) return fail(EMPI_ERR_INVALID_ARGUMENT, "pairsNotCollected");
    empi_status st = set_device(b->eng);
    if (st != EMPI_OK) return st;
    const int iters = b->settings.iteration_max;
    std::vector<InstState> sts(b->insts.size());
    std::vector<int4> ind((size_t)b->insts.size() * iters);
    CUDA_TRY(cudaMemcpy(sts.data(), b->d_state.p, sizeof(InstState) * sts.size(), cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(ind.data(), b->d_indices.p, sizeof(int4) * ind.size(), cudaMemcpyDeviceToHost));
    int n = 0;
    for (size_t i = 0; i < b->insts.size(); ++i) {
        const DictPlan& dp = b->dicts[b->insts[i].dict];
        for (int a = 0; a < sts[i].it; ++a, ++n) {
            if (n >= cap) continue;
            const int4 v = ind[i * iters + a];
            const ScalePlan& sp = b->scales[dp.scale0 + v.x];
            // the chosen atom's block: scale band x time tile (kernels.cuh, block proposal)
            block[n] = (v.x * kPropBands / dp.nscales) * kPropTiles + (int)((long long)kPropTiles * v.y / sp.tcount);
            CUDA_TRY(cudaMemcpy(spec + (size_t)n * kSpecSize, b->d_pairs.p + (i * iters + a) * (size_t)kSpecSize,
                                sizeof(float) * kSpecSize, cudaMemcpyDeviceToHost));
        }
    }
    *count = n;
    return ok();
}

extern "C" empi_status empi_batch_tree(empi_batch* b, int instance, long long slot_cap, unsigned long long* slots,
                                       long long* slot_count, int chunk_cap, unsigned long long* chunks,
                                       unsigned* chunk_l, int* chunk_count) {
    if (!b || !slot_count || !chunk_count || instance < 0 || instance >= (int)b->insts.size())
        return fail(EMPI_ERR_INVALID_ARGUMENT, "invalidArgument");
    const InstPlan& ip = b->insts[instance];
    const DictPlan& dp = b->dicts[ip.dict];
    *slot_count = dp.slots;
    *chunk_count = dp.chunks;
    if (!slots && !chunks && !chunk_l) return ok();
    if ((slots && slot_cap < dp.slots) || ((chunks || chunk_l) && chunk_cap < dp.chunks))
        return fail(EMPI_ERR_INVALID_ARGUMENT, "invalidArgument");
    empi_status st = set_device(b->eng);
    if (st != EMPI_OK) return st;
    if (slots)
        CUDA_TRY(cudaMemcpy(slots, b->d_slots.p + ip.slot_off, sizeof(unsigned long long) * dp.slots,
                            cudaMemcpyDeviceToHost));
    if (chunks)
        CUDA_TRY(cudaMemcpy(chunks, b->d_chunks.p + ip.chunk_off, sizeof(unsigned long long) * dp.chunks,
                            cudaMemcpyDeviceToHost));
    if (chunk_l)
        CUDA_TRY(cudaMemcpy(chunk_l, b->d_chunk_l.p + ip.chunk_off, sizeof(unsigned) * dp.chunks,
                            cudaMemcpyDeviceToHost));
    return ok();
}

namespace {
empi_status on_device(int device) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return fail(EMPI_ERR_NO_DEVICE, "noCudaDevice");
    if (device < 0 || device >= n) return fail(EMPI_ERR_INVALID_ARGUMENT, "invalidDevice");
    CUDA_TRY(cudaSetDevice(device));
    return EMPI_OK;
}
}  // namespace

extern "C" empi_status empi_proposal_scores(int device, const float* spec, int n, const float* weights, int bf16,
                                            float* scores) {
    if (!spec || !weights || !scores || n < 0) return fail(EMPI_ERR_INVALID_ARGUMENT, "invalidArgument");
    empi_status st = on_device(device);
    if (st != EMPI_OK) return st;
    std::string err;
    if (!net_scores(spec, n, weights, bf16, scores, &err)) return fail(EMPI_ERR_CUDA, err);
    return ok();
}

extern "C" empi_status empi_proposal_gradients(int device, const float* spec, const int* labels, int n,
                                               const float* weights, float* grads, float* loss) {
    if (!spec || !labels || !weights || !grads || !loss || n <= 0)
        return fail(EMPI_ERR_INVALID_ARGUMENT, "invalidArgument");
    for (int i = 0; i < n; ++i)
        if (labels[i] < 0 || labels[i] >= kProposalBlocks) return fail(EMPI_ERR_INVALID_ARGUMENT, "invalidLabel");
    empi_status st = on_device(device);
    if (st != EMPI_OK) return st;
    std::string err;
    if (!net_gradients(spec, labels, n, weights, grads, loss, &err)) return fail(EMPI_ERR_CUDA, err);
    return ok();
}

extern "C" empi_status empi_proposal_train(int device, const float* spec, const int* labels, int n, int epochs,
                                           int batch, float lr, float momentum, unsigned seed, float* weights,
                                           float* losses) {
    if (!spec || !labels || !weights || n <= 0 || epochs <= 0 || batch <= 0)
        return fail(EMPI_ERR_INVALID_ARGUMENT, "invalidArgument");
    for (int i = 0; i < n; ++i)
        if (labels[i] < 0 || labels[i] >= kProposalBlocks) return fail(EMPI_ERR_INVALID_ARGUMENT, "invalidLabel");
    empi_status st = on_device(device);
    if (st != EMPI_OK) return st;
    std::string err;
    if (!net_train(spec, labels, n, epochs, batch, lr, momentum, seed, weights, losses, &err))
        return fail(EMPI_ERR_CUDA, err);
    return ok();
}

extern "C" int empi_proposal_parameter_count(void) { return kNetParams; }

extern "C" empi_status empi_batch_probe_proposal(empi_batch* b, int enable) {
    if (!b) return fail(EMPI_ERR_INVALID_ARGUMENT, "invalidArgument");
    empi_status st = set_device(b->eng);
    if (st != EMPI_OK) return st;
    CUDA_TRY(cudaStreamSynchronize(b->eng->stream));
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    if (enable && b->dev.prange) return fail(EMPI_ERR_INVALID_ARGUMENT, "proposalWithProbe");
    if (enable) {
        if (!b->d_prop.p) CUDA_TRY(b->d_prop.alloc(b->d_slots.n));
        if (!b->d_probe.p) CUDA_TRY(b->d_probe.alloc(4));
        b->dev.prop = b->d_prop.p;
        b->dev.probe = b->d_probe.p;
    } else {
        b->dev.prop = nullptr;
        b->dev.probe = nullptr;
    }
    return ok();
}

namespace {

// the last run's results on the host, copied once per run (empi_batch_atoms
// and empi_batch_total_energy read every epoch from this copy)
empi_status fetch_results(empi_batch* b) {
    if (b->hm.valid) return EMPI_OK;
    auto& h = b->hm;
    h.st.resize(b->insts.size());
    h.en.resize(b->d_energies.n);
    h.ind.resize(b->d_indices.n);
    h.atoms.resize(b->d_atoms.n);
    h.fit.resize(b->d_fit_atoms.n);
    CUDA_TRY(cudaMemcpy(h.st.data(), b->d_state.p, sizeof(InstState) * h.st.size(), cudaMemcpyDeviceToHost));
    if (!h.en.empty())
        CUDA_TRY(cudaMemcpy(h.en.data(), b->d_energies.p, sizeof(double) * h.en.size(), cudaMemcpyDeviceToHost));
    if (!h.ind.empty())
        CUDA_TRY(cudaMemcpy(h.ind.data(), b->d_indices.p, sizeof(int4) * h.ind.size(), cudaMemcpyDeviceToHost));
    if (!h.atoms.empty())
        CUDA_TRY(cudaMemcpy(h.atoms.data(), b->d_atoms.p, sizeof(double) * h.atoms.size(), cudaMemcpyDeviceToHost));
    if (!h.fit.empty())
        CUDA_TRY(cudaMemcpy(h.fit.data(), b->d_fit_atoms.p, sizeof(double) * h.fit.size(), cudaMemcpyDeviceToHost));
    h.valid = true;
    return EMPI_OK;
}

}  // namespace

extern "C" empi_status empi_batch_atoms(empi_batch* b, int epoch, int cap, double* atoms, int* count,
                                        double* energies, int* indices) {
    if (!b || epoch < 0 || epoch >= (int)b->epochs.size() || cap < 0 || (cap > 0 && !atoms))
        return fail(EMPI_ERR_INVALID_ARGUMENT, "invalidArgument");
    empi_status st = set_device(b->eng);
    if (st != EMPI_OK) return st;
    st = fetch_results(b);
    if (st != EMPI_OK) return st;
    const auto& h = b->hm;
    const int C = b->epochs[epoch].channels;
    const int iters = b->settings.iteration_max;
    const int i0 = b->epoch_first_inst[epoch];
    const InstPlan& ip0 = b->insts[i0];
    const InstState* sts = h.st.data() + i0;
    const double* en = h.en.data() + (size_t)i0 * iters;
    const int4* ind = h.ind.data() + (size_t)i0 * iters;
    const int lim = std::min(cap, iters);
    if (ip0.chan0 >= 0) {  // SMP: one loop per channel
        for (int c = 0; c < C; ++c) {
            const InstPlan& ip = b->insts[i0 + c];
            const int n = std::min(sts[c].it, lim);
            if (count) count[c] = sts[c].it;
            if (n > 0)
                std::memcpy(atoms + (size_t)c * cap * 6, h.atoms.data() + ip.out_off, sizeof(double) * 6 * n);
            for (int a = 0; a < lim; ++a) {
                if (energies) energies[(size_t)c * cap + a] = en[(size_t)c * iters + a];
                if (indices) {
                    const int4 v = ind[(size_t)c * iters + a];
                    indices[((size_t)c * cap + a) * 3] = v.x;
                    indices[((size_t)c * cap + a) * 3 + 1] = v.y;
                    indices[((size_t)c * cap + a) * 3 + 2] = v.z;
                }
            }
        }
    } else {
        const int n = std::min(sts[0].it, lim);
        if (count)
            for (int c = 0; c < C; ++c) count[c] = sts[0].it;
        if (ip0.chan0 == -2) {  // MMP2: per-channel fits
            const int f0 = b->epoch_first_fit[epoch];
            for (int c = 0; c < C; ++c)
                if (n > 0)
                    std::memcpy(atoms + (size_t)c * cap * 6, h.fit.data() + ((size_t)(f0 + c) * iters) * 6,
                                sizeof(double) * 6 * n);
        } else {
            const double* src = h.atoms.data() + ip0.out_off;  // [a][c][6]
            for (int a = 0; a < n; ++a)
                for (int c = 0; c < C; ++c)
                    std::memcpy(atoms + ((size_t)c * cap + a) * 6, src + ((size_t)a * C + c) * 6, sizeof(double) * 6);
        }
        for (int a = 0; a < lim; ++a) {
            if (energies) energies[a] = en[a];
            if (indices) {
                indices[a * 3] = ind[a].x;
                indices[a * 3 + 1] = ind[a].y;
                indices[a * 3 + 2] = ind[a].z;
            }
        }
    }
    return ok();
}

extern "C" empi_status empi_batch_total_energy(empi_batch* b, int epoch, double* totals) {
    if (!b || !totals || epoch < 0 || epoch >= (int)b->epochs.size())
        return fail(EMPI_ERR_INVALID_ARGUMENT, "invalidArgument");
    empi_status st = set_device(b->eng);
    if (st != EMPI_OK) return st;
    st = fetch_results(b);
    if (st != EMPI_OK) return st;
    const int i0 = b->epoch_first_inst[epoch];
    const int n = b->insts[i0].chan0 >= 0 ? b->epochs[epoch].channels : 1;
    for (int i = 0; i < n; ++i) totals[i] = b->hm.st[i0 + i].etotal;
    return ok();
}

extern "C" empi_status empi_batch_get_stats(empi_batch* b, empi_batch_stats* out) {
    if (!b || !out) return fail(EMPI_ERR_INVALID_ARGUMENT, "invalidArgument");
    *out = b->stats;
    return ok();
}

extern "C" empi_status empi_decompose(empi_engine* eng, empi_variant variant, const empi_dictionary* dict,
                                      const empi_settings* settings, const empi_epoch* epochs, int count, int cap,
                                      double* atoms, int* counts) {
    empi_batch* b = nullptr;
    empi_status st = empi_batch_create(eng, variant, dict, settings, epochs, count, &b);
    if (st != EMPI_OK) return st;
    std::unique_ptr<empi_batch, void (*)(empi_batch*)> guard(b, empi_batch_destroy);
    st = empi_batch_load(b, epochs);
    if (st != EMPI_OK) return st;
    st = empi_batch_run(b);
    if (st != EMPI_OK) return st;
    size_t off = 0, coff = 0;
    for (int e = 0; e < count; ++e) {
        st = empi_batch_atoms(b, e, cap, atoms ? atoms + off : nullptr, counts ? counts + coff : nullptr, nullptr,
                              nullptr);
        if (st != EMPI_OK) return st;
        off += (size_t)epochs[e].channels * cap * 6;
        coff += epochs[e].channels;
    }
    return ok();
}

// ------------------------------------------------------------ workspace seam

struct empi_workspace {
    empi_batch* b = nullptr;
    int C = 0, N = 0;
    double fs = 0;
    double* d_params = nullptr;
    ~empi_workspace() {
        if (d_params) cudaFree(d_params);
        if (b) empi_batch_destroy(b);
    }
};

namespace {

empi_status ws_reset_state(empi_workspace* w) {
    empi_batch* b = w->b;
    cudaStream_t s = b->eng->stream;
    CUDA_TRY(cudaMemset2DAsync(b->d_state.p, sizeof(InstState), 0, 4 * sizeof(int), b->insts.size(), s));
    CUDA_TRY(cudaMemsetAsync(b->d_ctr.p + CTR_CSLOTS, 0, sizeof(int) * 4, s));
    CUDA_TRY(cudaMemsetAsync(b->d_ctr.p + CTR_STALLED, 0, sizeof(int), s));
    return EMPI_OK;
}

}  // namespace

extern "C" empi_status empi_workspace_create(empi_engine* eng, const empi_dictionary* dict, double fs, int channels,
                                             int samples, empi_variant variant, empi_workspace** out) {
    if (!eng || !dict || !out || channels <= 0) return fail(EMPI_ERR_INVALID_ARGUMENT, "invalidArgument");
    *out = nullptr;
    std::unique_ptr<empi_workspace> w(new empi_workspace);
    empi_epoch ep{fs, channels, samples, nullptr};
    empi_settings set{1, 0.0};
    const int v = channels == 1 ? EMPI_SMP : (variant == EMPI_MMP1 ? EMPI_MMP1 : EMPI_MMP3);
    empi_status st = build_batch(eng, v, dict, &set, &ep, 1, 1, &w->b);
    if (st != EMPI_OK) return st;
    w->C = channels;
    w->N = samples;
    w->fs = fs;
    CUDA_TRY(cudaMalloc(&w->d_params, sizeof(double) * 6 * channels));
    *out = w.release();
    return ok();
}

extern "C" void empi_workspace_destroy(empi_workspace* w) { delete w; }

extern "C" empi_status empi_workspace_compute(empi_workspace* w, const double* samples) {
    if (!w || !samples) return fail(EMPI_ERR_INVALID_ARGUMENT, "invalidArgument");
    empi_batch* b = w->b;
    empi_status st = set_device(b->eng);
    if (st != EMPI_OK) return st;
    cudaStream_t s = b->eng->stream;
    CUDA_TRY(cudaMemcpyAsync(b->d_residual.p, samples, sizeof(double) * (size_t)w->C * w->N, cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaMemsetAsync(b->d_ctr.p, 0, sizeof(int) * CTR_COUNT, s));
    k_init<<<(int)b->blk_ic.size(), 256, 0, s>>>(b->dev, 0);
    launch_update(b, SCHED_INIT, -1, 0.0, 0.0, s, nullptr, nullptr);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(s));
    return ok();
}

extern "C" empi_status empi_workspace_find_best(empi_workspace* w, double* params, int* index) {
    if (!w || !params) return fail(EMPI_ERR_INVALID_ARGUMENT, "invalidArgument");
    empi_batch* b = w->b;
    empi_status st = set_device(b->eng);
    if (st != EMPI_OK) return st;
    cudaStream_t s = b->eng->stream;
    for (;;) {
        st = ws_reset_state(w);
        if (st != EMPI_OK) return st;
        launch_select(b, s);
        CUDA_TRY(cudaGetLastError());
        InstState is;
        CUDA_TRY(cudaMemcpyAsync(&is, b->d_state.p, sizeof(is), cudaMemcpyDeviceToHost, s));
        CUDA_TRY(cudaStreamSynchronize(s));
        if (is.status != ST_STALLED) break;
        // more candidates than the buffers hold: grow them and select again
        if (b->regrows >= 12) return fail(EMPI_ERR_CANDIDATE_OVERFLOW, "candidateOverflow");
        st = grow_candidates(b);
        if (st != EMPI_OK) return st;
    }
    st = check_errors(b);
    if (st != EMPI_OK) return st;
    CUDA_TRY(cudaMemcpy(params, b->d_atoms.p, sizeof(double) * 6 * w->C, cudaMemcpyDeviceToHost));
    if (index) {
        int4 v;
        CUDA_TRY(cudaMemcpy(&v, b->d_indices.p, sizeof(int4), cudaMemcpyDeviceToHost));
        index[0] = v.x;
        index[1] = v.y;
        index[2] = v.z;
    }
    return ok();
}

extern "C" empi_status empi_workspace_atom_count(const empi_workspace* w, uint64_t* count) {
    if (!w || !count) return fail(EMPI_ERR_INVALID_ARGUMENT, "invalidArgument");
    *count = w->b->dicts[0].values;
    return ok();
}

extern "C" empi_status empi_workspace_subtract_atom(empi_workspace* w, const double* params, double* samples,
                                                    int channel) {
    if (!w || !params || !samples || channel < 0 || channel >= w->C)
        return fail(EMPI_ERR_INVALID_ARGUMENT, "invalidArgument");
    empi_batch* b = w->b;
    empi_status st = set_device(b->eng);
    if (st != EMPI_OK) return st;
    cudaStream_t s = b->eng->stream;
    double* x = b->d_residual.p + (size_t)channel * w->N;
    CUDA_TRY(cudaMemcpyAsync(x, samples, sizeof(double) * w->N, cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaMemcpyAsync(w->d_params, params, sizeof(double) * 6, cudaMemcpyHostToDevice, s));
    k_subtract_signal<<<1, 256, 0, s>>>(x, b->d_residual32.p + (size_t)channel * w->N, w->N, w->fs, w->d_params, 0);
    CUDA_TRY(cudaMemcpyAsync(samples, x, sizeof(double) * w->N, cudaMemcpyDeviceToHost, s));
    st = ws_reset_state(w);
    if (st != EMPI_OK) return st;
    // src/gabor.cpp:189-209: refresh every window within 3 (s + sA) of tA
    launch_update(b, SCHED_ATOM, -1, params[2] / w->fs, params[3] / w->fs, s, nullptr, nullptr);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(s));
    return ok();
}

extern "C" empi_status empi_workspace_energy_map(empi_workspace* w, int scale, float* energy) {
    if (!w || !energy) return fail(EMPI_ERR_INVALID_ARGUMENT, "invalidArgument");
    empi_batch* b = w->b;
    if (scale < 0 || scale >= b->dicts[0].nscales) return fail(EMPI_ERR_INVALID_ARGUMENT, "invalidScale");
    empi_status st = set_device(b->eng);
    if (st != EMPI_OK) return st;
    const ScalePlan& sp = b->scales[scale];
    const size_t n = (size_t)sp.fcount * sp.tcount;
    DevBuf<float> dump;
    CUDA_TRY(dump.alloc(n));
    cudaStream_t s = b->eng->stream;
    CUDA_TRY(cudaMemsetAsync(dump.p, 0, sizeof(float) * n, s));
    st = ws_reset_state(w);
    if (st != EMPI_OK) return st;
    b->dev.dump = dump.p;
    launch_update(b, SCHED_INIT, scale, 0.0, 0.0, s, nullptr, nullptr);
    b->dev.dump = nullptr;
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(energy, dump.p, sizeof(float) * n, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    return ok();
}

extern "C" empi_status empi_subtract_atom_from_signal(empi_engine* eng, double* params, double* samples, int n,
                                                      double fs, int fit) {
    if (!eng || !params || !samples || n <= 0 || !(fs > 0)) return fail(EMPI_ERR_INVALID_ARGUMENT, "invalidArgument");
    empi_status st = set_device(eng);
    if (st != EMPI_OK) return st;
    DevBuf<double> x, p;
    CUDA_TRY(x.alloc(n));
    CUDA_TRY(p.alloc(6));
    cudaStream_t s = eng->stream;
    CUDA_TRY(cudaMemcpyAsync(x.p, samples, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaMemcpyAsync(p.p, params, sizeof(double) * 6, cudaMemcpyHostToDevice, s));
    k_subtract_signal<<<1, 256, 0, s>>>(x.p, nullptr, n, fs, p.p, fit);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(samples, x.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaMemcpyAsync(params, p.p, sizeof(double) * 6, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    return ok();
}

// ------------------------------------------------------------ allocation-free subtraction

// Device copy of the signal (EMPI_NOALLOC_MAX_SAMPLES doubles) followed by the
// six atom params, for empi_subtract_atom_from_signal_noalloc.  It is a fixed
// static array so callers that may not allocate (a device whose memory another
// framework's pool owns, a fixed device-memory budget) can still run the
// subtraction; every device that loads the library holds these 8 MiB until
// exit.
static __device__ __align__(256) double g_subtract_staging[EMPI_NOALLOC_MAX_SAMPLES + 8];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_staging_mutex;
// device address of the array, per device, looked up on the first call with
// that device current (a later cudaDeviceReset of the device is unsupported)
double* g_staging_ptr[kMaxDevices] = {};
}  // namespace

extern "C" empi_status empi_subtract_atom_from_signal_noalloc(int device, void* stream, double* params,
                                                              double* samples, int n, double fs, int fit) {
    if (!params || !samples || !(fs > 0) || n <= 0) return fail(EMPI_ERR_INVALID_ARGUMENT, "invalidArgument");
    if (n > EMPI_NOALLOC_MAX_SAMPLES) return fail(EMPI_ERR_INVALID_ARGUMENT, "signalLongerThanStaticScratch");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return fail(EMPI_ERR_NO_DEVICE, "noCudaDevice");
    if (device < 0 || device >= count || device >= kMaxDevices) return fail(EMPI_ERR_INVALID_ARGUMENT, "invalidDevice");
    int prev = 0;
    CUDA_TRY(cudaGetDevice(&prev));
    CUDA_TRY(cudaSetDevice(device));
    double* base = nullptr;
    {
        // set-up once per device, with that device current: in host code the
        // array's name is only a stand-in, the kernel needs its device address
        std::lock_guard<std::mutex> lock(g_staging_mutex);
        if (!g_staging_ptr[device]) {
            double* p = nullptr;
            cudaError_t ce = cudaGetSymbolAddress((void**)&p, g_subtract_staging);
            if (ce != cudaSuccess || !p) {
                cudaSetDevice(prev);
                return fail(EMPI_ERR_CUDA, std::string("cuda: ") + cudaGetErrorString(ce) + " (staging address)");
            }
            g_staging_ptr[device] = p;
        }
        base = g_staging_ptr[device];
    }
    double* x = base;
    double* prm = base + EMPI_NOALLOC_MAX_SAMPLES;
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t ce = cudaMemcpyAsync(x, samples, sizeof(double) * (size_t)n, cudaMemcpyHostToDevice, s);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(prm, params, sizeof(double) * 6, cudaMemcpyHostToDevice, s);
    if (ce == cudaSuccess) {
        k_subtract_signal<<<1, 256, 0, s>>>(x, nullptr, n, fs, prm, fit);
        ce = cudaGetLastError();
    }
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(samples, x, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost, s);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(params, prm, sizeof(double) * 6, cudaMemcpyDeviceToHost, s);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
    cudaSetDevice(prev);
    if (ce != cudaSuccess) return fail(EMPI_ERR_CUDA, std::string("cuda: ") + cudaGetErrorString(ce));
    return ok();
}
