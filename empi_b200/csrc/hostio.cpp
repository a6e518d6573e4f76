// Host surface kept from empi: the key/value config file, the float32 signal
// reader, the SVAROG (MPv5) book writer and the CLI driver with its stdout
// progress protocol.  Epochs stream through the device in batches, the next
// batch read from the file while the current one decomposes.
#include <algorithm>
#include <atomic>
#include <cctype>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <map>
#include <mutex>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/empi_b200.h"
#include "engine.hpp"

namespace {

constexpr int kStreamEpochs = 64;  // epochs per device batch unless the config says otherwise

struct Error : std::runtime_error {
    empi_status status;
    Error(empi_status st, const std::string& m) : std::runtime_error(m), status(st) {}
};

// ------------------------------------------------------------ configuration

// Configuration::parse/has/at, src/conf.cpp:10-48: "name<ws>value" lines,
// '#' starts a comment line, the value runs to the end of the line.
class Configuration {
    std::map<std::string, std::string> values;

public:
    void parse(const std::string& path) {
        std::ifstream stream(path);
        if (!stream) throw Error(EMPI_ERR_CONFIG, "couldNotOpenConfigFile");
        values.clear();
        std::string line;
        while (std::getline(stream, line)) {
            std::string::size_type iname = line.find_first_not_of(" \t");
            if (iname == std::string::npos || line[iname] == '#') continue;
            std::string::size_type ispace = line.find_first_of(" \t", iname + 1);
            if (ispace == std::string::npos) continue;
            std::string::size_type ivalue = line.find_first_not_of(" \t", ispace + 1);
            if (ivalue == std::string::npos) continue;
            std::string name = line.substr(iname, ispace - iname);
            std::string value = line.substr(ivalue);
            if (!name.empty() && !value.empty()) values[name] = value;
        }
    }
    bool has(const std::string& key) const { return values.count(key) != 0; }
    const std::string& at(const std::string& key) const {
        auto it = values.find(key);
        if (it == values.end()) throw Error(EMPI_ERR_CONFIG, "missingConfigurationEntry:" + key);
        return it->second;
    }
};

// parseIntegerSubset, src/empi.cpp:22-47 ("1-3,5")
std::vector<int> parse_subset(const std::string& text, int max) {
    std::stringstream ss(text);
    std::string item;
    std::vector<int> numbers;
    while (std::getline(ss, item, ',')) {
        int start, end;
        int status = sscanf(item.c_str(), "%d-%d", &start, &end);
        if (status == 2 && start >= 1 && end <= max) {
            for (int i = start; i <= end; ++i) numbers.push_back(i);
        } else if (status == 1 && start >= 1 && start <= max) {
            numbers.push_back(start);
        } else {
            throw Error(EMPI_ERR_CONFIG, "invalidSubsetSpecification");
        }
    }
    if (numbers.empty()) throw Error(EMPI_ERR_CONFIG, "emptySubsetSpecification");
    return numbers;
}

// ------------------------------------------------------------ signal reader

// SignalReader and its three modes, src/io.cpp:9-85.  Samples are float32,
// channels interleaved; the selected channels are kept (1-based).
class SignalReader {
    FILE* file = nullptr;
    int mode = 0;  // 0 all epochs, 1 selected epochs, 2 whole signal
    int epochSize = 0;
    std::vector<int> epochs;
    size_t nextEpoch = 0;
    bool wholeDone = false;

public:
    std::string path;
    int channelCount = 0;
    double freqSampling = 0;
    std::vector<int> selectedChannels;

    SignalReader(const std::string& p, int mode_, int epochSize_, std::vector<int> epochs_)
        : mode(mode_), epochSize(epochSize_), epochs(std::move(epochs_)), path(p) {
        file = fopen(p.c_str(), "rb");
        if (!file) throw Error(EMPI_ERR_IO, "couldNotOpenSignalFile");
    }
    ~SignalReader() {
        if (file) fclose(file);
    }

    // returns samples x C (selected channels), interleaved; empty at the end
    std::vector<float> readEpoch(long samplesToRead, int& count) {
        const int C = (int)selectedChannels.size();
        std::vector<float> out;
        std::vector<float> frame(channelCount);
        long left = INT_MAX;
        count = 0;
        while (samplesToRead-- > 0 &&
               fread(frame.data(), sizeof(float), channelCount, file) == (size_t)channelCount) {
            if (--left < 0) throw Error(EMPI_ERR_IO, "signalFileIsTooLongForThisMachine");
            for (int i = 0; i < C; ++i) out.push_back(frame[selectedChannels[i] - 1]);
            ++count;
        }
        return out;
    }

    std::vector<float> read(int& count) {
        if (mode == 0) {
            std::vector<float> r = readEpoch(epochSize, count);
            if (count > 0 && count != epochSize) throw Error(EMPI_ERR_IO, "fileIsTruncated");
            return r;
        }
        if (mode == 1) {
            if (nextEpoch >= epochs.size()) {
                count = 0;
                return {};
            }
            int epoch = epochs[nextEpoch++];
            if (fseek(file, (long)sizeof(float) * channelCount * (long)epochSize * (epoch - 1), SEEK_SET))
                throw Error(EMPI_ERR_IO, "signalSeekFailed");
            std::vector<float> r = readEpoch(epochSize, count);
            if (count != epochSize) throw Error(EMPI_ERR_IO, "fileIsTruncated");
            return r;
        }
        if (wholeDone) {
            count = 0;
            return {};
        }
        wholeDone = true;
        return readEpoch(INT_MAX, count);
    }
};

// ------------------------------------------------------------ book writer

// Big-endian encoders (inc/io.hpp:18-61)
void put_u8(std::vector<uint8_t>& b, unsigned v) { b.push_back((uint8_t)v); }
void put_u16(std::vector<uint8_t>& b, unsigned v) {
    b.push_back((uint8_t)(v >> 8));
    b.push_back((uint8_t)v);
}
void put_u32(std::vector<uint8_t>& b, uint32_t v) {
    b.push_back((uint8_t)(v >> 24));
    b.push_back((uint8_t)(v >> 16));
    b.push_back((uint8_t)(v >> 8));
    b.push_back((uint8_t)v);
}
void put_f32(std::vector<uint8_t>& b, double v) {
    float f = (float)v;
    uint32_t u;
    std::memcpy(&u, &f, 4);
    put_u32(b, u);
}
void set_u32(std::vector<uint8_t>& b, size_t at, uint32_t v) {
    b[at] = (uint8_t)(v >> 24);
    b[at + 1] = (uint8_t)(v >> 16);
    b[at + 2] = (uint8_t)(v >> 8);
    b[at + 3] = (uint8_t)v;
}

// MPv5 header: version, comment "empi", signal and decomposition info with the
// constant fields of src/io.cpp:111-117 (inc/io.hpp:65-98 layout).
void book_header(std::vector<uint8_t>& b, int C, double fs) {
    const char version[6] = {'M', 'P', 'v', '5', '.', '0'};
    b.insert(b.end(), version, version + 6);
    put_u8(b, 1);
    put_u32(b, 4);
    const char comment[4] = {'e', 'm', 'p', 'i'};
    b.insert(b.end(), comment, comment + 4);
    put_u8(b, 2);
    put_u32(b, 27);
    put_u8(b, 5);
    put_u8(b, 10);
    put_f32(b, fs);
    put_f32(b, 1.0);   // pointsPerMicrovolt
    put_u16(b, (unsigned)C);
    put_u8(b, 6);
    put_u8(b, 13);
    put_f32(b, 100.0); // energyPercent
    put_u32(b, 1);     // iterationCount
    put_u32(b, 0);     // dictionarySize
    put_u8(b, 'F');
}

// One epoch block (BookWriter::write, src/io.cpp:119-167): signal and atoms
// per channel, with lengths patched after the fact.
void book_epoch(std::vector<uint8_t>& b, int epochNumber, int C, int N, const float* samples, int cap,
                const double* atoms, const int* counts) {
    const size_t dataPos = b.size();
    put_u8(b, 7);
    put_u32(b, 0);
    put_u16(b, (unsigned)epochNumber);
    put_u32(b, (uint32_t)N);
    for (int c = 0; c < C; ++c) {
        put_u8(b, 8);
        put_u32(b, (uint32_t)(2 + 4 * (size_t)N));
        put_u16(b, (unsigned)(c + 1));
        for (int i = 0; i < N; ++i) put_f32(b, samples[(size_t)c * N + i]);
        const size_t atomsPos = b.size();
        put_u8(b, 9);
        put_u32(b, 0);
        put_u16(b, (unsigned)(c + 1));
        const int n = std::min(counts[c], cap);
        for (int a = 0; a < n; ++a) {
            put_u8(b, 13);  // ATOM_GABOR
            put_u8(b, 24);  // six float32 params
            for (int p = 0; p < 6; ++p) put_f32(b, atoms[((size_t)c * cap + a) * 6 + p]);
        }
        set_u32(b, atomsPos + 1, (uint32_t)(b.size() - atomsPos - 5));
    }
    set_u32(b, dataPos + 1, (uint32_t)(b.size() - dataPos - 5));
}

void write_file(const std::string& path, const std::vector<uint8_t>& bytes, bool append) {
    FILE* f = fopen(path.c_str(), append ? "ab" : "wb");
    if (!f) throw Error(EMPI_ERR_IO, "couldNotCreateOutputFile");
    if (!bytes.empty() && fwrite(bytes.data(), 1, bytes.size(), f) != bytes.size()) {
        fclose(f);
        throw Error(EMPI_ERR_IO, "couldNotWriteOutputFile");
    }
    fclose(f);
}

void check(empi_status st) {
    if (st != EMPI_OK) throw Error(st, empi_last_error()[0] ? empi_last_error() : empi_status_string(st));
}

// The empi() body, src/empi.cpp:49-167.
void run_config(const char* configPath, const empi_engine_opts* opts) {
    Configuration conf;
    conf.parse(configPath);
    const double energyError = atof(conf.at("energyError").c_str());
    if (energyError <= 0.0 || energyError >= 1.0) throw Error(EMPI_ERR_CONFIG, "invalidEnergyErrorValue");
    empi_dictionary dict;
    dict.energy_error = energyError;
    dict.scale_min = conf.has("minAtomScale") ? atof(conf.at("minAtomScale").c_str()) : 0.0;
    dict.scale_max = conf.has("maxAtomScale") ? atof(conf.at("maxAtomScale").c_str()) : INFINITY;
    dict.freq_max = conf.has("maxAtomFrequency") ? atof(conf.at("maxAtomFrequency").c_str()) : INFINITY;
    empi_settings settings;
    settings.iteration_max = atoi(conf.at("maximalNumberOfIterations").c_str());
    if (settings.iteration_max <= 0) throw Error(EMPI_ERR_CONFIG, "invalidMaximalNumberOfIterations");
    settings.residual_energy = 1 - 0.01 * atof(conf.at("energyPercent").c_str());
    if (settings.residual_energy < 0 || settings.residual_energy >= 1.0)
        throw Error(EMPI_ERR_CONFIG, "invalidEnergyPercentValue");

    const std::string& signalPath = conf.at("nameOfDataFile");
    std::unique_ptr<SignalReader> reader;
    if (conf.has("numberOfSamplesInEpoch")) {
        int epochSize = atoi(conf.at("numberOfSamplesInEpoch").c_str());
        if (epochSize <= 0) throw Error(EMPI_ERR_CONFIG, "invalidNumberOfSamplesInEpoch");
        if (conf.has("selectedEpochs")) {
            std::vector<int> epochs = parse_subset(conf.at("selectedEpochs"), INT_MAX / epochSize);
            reader.reset(new SignalReader(signalPath, 1, epochSize, epochs));
        } else {
            reader.reset(new SignalReader(signalPath, 0, epochSize, {}));
        }
    } else {
        if (conf.has("selectedEpochs")) conf.at("numberOfSamplesInEpoch");
        reader.reset(new SignalReader(signalPath, 2, 0, {}));
    }
    reader->freqSampling = atof(conf.at("samplingFrequency").c_str());
    if (reader->freqSampling <= 0.0) throw Error(EMPI_ERR_CONFIG, "invalidSamplingFrequency");
    reader->channelCount = atoi(conf.at("numberOfChannels").c_str());
    if (reader->channelCount <= 0) throw Error(EMPI_ERR_CONFIG, "invalidNumberOfChannels");
    reader->selectedChannels = parse_subset(conf.at("selectedChannels"), reader->channelCount);

    const int C = (int)reader->selectedChannels.size();
    std::string typeOfMP = conf.at("MP");
    std::transform(typeOfMP.begin(), typeOfMP.end(), typeOfMP.begin(), ::tolower);
    empi_variant variant;
    if (C == 1 || typeOfMP == "smp") variant = EMPI_SMP;
    else if (typeOfMP == "mmp1") variant = EMPI_MMP1;
    else if (typeOfMP == "mmp2") variant = EMPI_MMP2;
    else if (typeOfMP == "mmp3") variant = EMPI_MMP3;
    else throw Error(EMPI_ERR_CONFIG, "unsupportedDecompositionType");

    std::string prefix = reader->path;
    std::string::size_type slash = prefix.find_last_of('/');
    if (slash != std::string::npos) prefix = prefix.substr(slash + 1);
    prefix = prefix.substr(0, prefix.find_last_of('.'));
    typeOfMP.resize(3);
    const std::string bookPath = conf.at("nameOfOutputDirectory") + "/" + prefix + "_" + typeOfMP + ".b";
    write_file(bookPath, {}, false);  // BookWriter opens (truncates) the file up front

    // Epochs stream through the GPU in batches of gpuEpochsPerBatch (an
    // optional key the reference ignores; default kStreamEpochs): while one
    // batch decomposes on a worker thread, the next is read from the file, and
    // each batch's protocol lines and book blocks are written as soon as it
    // ends.  A read error ends the job after the epochs before it are
    // decomposed and written, as in the reference's epoch loop.
    int perBatch = conf.has("gpuEpochsPerBatch") ? atoi(conf.at("gpuEpochsPerBatch").c_str()) : kStreamEpochs;
    if (perBatch <= 0) throw Error(EMPI_ERR_CONFIG, "invalidGpuEpochsPerBatch");
    struct Chunk {
        std::vector<std::vector<float>> epochs;
        std::unique_ptr<Error> pending;  // read error after these epochs
    };
    int N = 0;
    auto readChunk = [&](Chunk& ch) {
        ch.epochs.clear();
        ch.pending.reset();
        try {
            while ((int)ch.epochs.size() < perBatch) {
                int count = 0;
                std::vector<float> e = reader->read(count);
                if (!count) break;
                if (N == 0) N = count;
                if (count != N) throw Error(EMPI_ERR_IO, "fileIsTruncated");
                ch.epochs.push_back(std::move(e));
            }
        } catch (const Error& e) {
            ch.pending.reset(new Error(e));
        }
    };

    // an autotuner cache (optional key the reference ignores): tuned launch
    // shapes for the workloads it holds
    empi_engine_opts eopts;
    empi_engine_opts_default(&eopts);
    if (opts) eopts = *opts;
    std::string tuneCache;
    if (conf.has("gpuTuneCache")) {
        tuneCache = conf.at("gpuTuneCache");
        eopts.tune_cache = tuneCache.c_str();
    }
    // GPUs: EMPI_DEVICES="0,1,..." shards every batch's epochs across one
    // engine per listed device (contiguous, equal shares: a batch's epochs
    // have one shape); otherwise the options' device
    std::vector<int> devices;
    if (const char* dv = getenv("EMPI_DEVICES")) {
        std::stringstream ds(dv);
        std::string tok;
        while (std::getline(ds, tok, ','))
            if (!tok.empty()) devices.push_back(atoi(tok.c_str()));
    }
    if (devices.empty()) devices.push_back(eopts.device);
    const int D = (int)devices.size();

    Chunk cur, next;
    readChunk(cur);
    std::vector<std::unique_ptr<empi_engine, void (*)(empi_engine*)>> eg;
    std::vector<std::unique_ptr<empi_batch, void (*)(empi_batch*)>> bg;
    for (int d = 0; d < D; ++d) {
        eg.emplace_back(nullptr, empi_engine_destroy);
        bg.emplace_back(nullptr, empi_batch_destroy);
    }
    std::vector<int> batchEpochs(D, 0);
    std::vector<char> staged(D, 0);  // a device's share of the current chunk is already on it
    uint64_t atomCount = 0;
    const int cap = settings.iteration_max;
    const bool smp = variant == EMPI_SMP;
    const int loops = smp ? C : 1;
    std::vector<float> chanMajor;
    int epochNumber = 0;
    while (!cur.epochs.empty()) {
        if (!eg[0]) {
            for (int d = 0; d < D; ++d) {
                empi_engine_opts o = eopts;
                o.device = devices[d];
                empi_engine* e = nullptr;
                check(empi_engine_create(&o, &e));
                eg[d].reset(e);
            }
            check(empi_dictionary_size(&dict, reader->freqSampling, N, &atomCount, nullptr));
            chanMajor.resize((size_t)C * N);
        }
        const int count = (int)cur.epochs.size();
        // device d takes epochs [first[d], first[d + 1])
        std::vector<int> first(D + 1);
        for (int d = 0; d <= D; ++d) first[d] = (int)((long long)count * d / D);
        auto owner = [&](int e) {
            int d = 0;
            while (first[d + 1] <= e) ++d;
            return d;
        };

        // The progress protocol (src/empi.cpp:159, src/classes.cpp:41-48,
        // 83) is printed in the reference's order -- epoch by epoch, MP loop
        // by loop -- as the devices advance: after every CUDA-graph chunk the
        // device holding the epoch being printed reports its atoms so far, and
        // the next loop starts printing once it is done.  Epochs of a batch
        // advance together, so the first epoch's lines follow the run step by
        // step.
        std::mutex printMutex;
        int pe = 0, pl = 0, pp = 0;
        bool startDone = false, chanDone = false;
        std::vector<double> en((size_t)cap);
        auto emit = [&](bool final, int fromDevice) {
            std::lock_guard<std::mutex> lock(printMutex);
            while (pe < count) {
                const int d = owner(pe);
                if (!final && d != fromDevice) return;  // its device's own hook prints it
                if (!startDone) {
                    std::cout << "START" << '\t' << (epochNumber + pe + 1) << '\t' << C << '\t'
                              << settings.iteration_max << '\t' << 100 * (1 - settings.residual_energy) << std::endl;
                    startDone = true;
                }
                if (smp && !chanDone) {
                    std::cout << "CHANNEL\t" << pl << std::endl;
                    chanDone = true;
                }
                int it = 0, running = 0;
                double total = 0.0;
                check(empi::batch_loop_progress(bg[d].get(), pe - first[d], pl, &it, &running, &total, en.data()));
                for (int k = pp + 1; k <= it; ++k) {
                    const double residue = k == 1 ? total : en[(size_t)k - 2];
                    const double energyProgress = 100.0 * (1.0 - residue / total);
                    const double totalProgress = std::max(100.0 * (k - 1) / settings.iteration_max, energyProgress);
                    std::cout << "ATOM\t" << (k - 1) << '\t' << atomCount << '\t' << energyProgress << '\t'
                              << totalProgress << std::endl;
                }
                pp = it;
                if (running && !final) return;
                pp = 0;
                chanDone = false;
                if (++pl == loops) {
                    pl = 0;
                    ++pe;
                    startDone = false;
                }
            }
        };

        // results of this batch, filled by the workers (one per device)
        std::vector<double> atoms((size_t)count * C * cap * 6);
        std::vector<int> counts((size_t)count * C);
        std::vector<std::exception_ptr> failure(D);
        std::atomic<bool> nextReady(false);
        std::vector<char> nextStaged(D, 0);
        std::vector<std::thread> workers;
        for (int d = 0; d < D; ++d) {
            const int n = first[d + 1] - first[d];
            if (n == 0) continue;
            workers.emplace_back([&, d, n] {
                try {
                    std::vector<empi_epoch> eps;
                    for (int e = first[d]; e < first[d + 1]; ++e)
                        eps.push_back(empi_epoch{reader->freqSampling, C, N, cur.epochs[e].data()});
                    if (!bg[d] || batchEpochs[d] != n) {
                        empi_batch* batch = nullptr;
                        bg[d].reset();
                        check(empi_batch_create(eg[d].get(), variant, &dict, &settings, eps.data(), n, &batch));
                        bg[d].reset(batch);
                        batchEpochs[d] = n;
                        staged[d] = 0;
                    }
                    if (!staged[d]) check(empi_batch_load(bg[d].get(), eps.data()));
                    check(empi::batch_run_hooked(bg[d].get(), [&] {
                        emit(false, d);
                        // this device's share of the next batch, copied on the
                        // copy stream while the rest of this run goes on
                        if (!nextStaged[d] && nextReady.load() && (int)next.epochs.size() == count && !next.pending) {
                            std::vector<empi_epoch> nx;
                            for (int e = first[d]; e < first[d + 1]; ++e)
                                nx.push_back(empi_epoch{reader->freqSampling, C, N, next.epochs[e].data()});
                            check(empi::batch_stage(bg[d].get(), nx.data()));
                            nextStaged[d] = 1;
                        }
                    }));
                    for (int e = 0; e < n; ++e)
                        check(empi_batch_atoms(bg[d].get(), e, cap, atoms.data() + (size_t)(first[d] + e) * C * cap * 6,
                                               counts.data() + (size_t)(first[d] + e) * C, nullptr, nullptr));
                } catch (...) {
                    failure[d] = std::current_exception();
                }
            });
        }
        if (!cur.pending) readChunk(next);  // overlaps the device runs
        nextReady.store(true);
        for (auto& t : workers) t.join();
        for (auto& f : failure)
            if (f) std::rethrow_exception(f);
        emit(true, -1);
        staged = nextStaged;

        std::vector<uint8_t> book;
        for (int e = 0; e < count; ++e) {
            ++epochNumber;
            const double* at = atoms.data() + (size_t)e * C * cap * 6;
            const int* cn = counts.data() + (size_t)e * C;
            for (int c = 0; c < C; ++c)
                for (int i = 0; i < N; ++i) chanMajor[(size_t)c * N + i] = cur.epochs[e][(size_t)i * C + c];
            if (epochNumber == 1) book_header(book, C, reader->freqSampling);
            book_epoch(book, epochNumber, C, N, chanMajor.data(), cap, at, cn);
        }
        write_file(bookPath, book, true);
        if (cur.pending) throw *cur.pending;
        std::swap(cur, next);
        next.epochs.clear();
    }
    if (cur.pending) throw *cur.pending;
    puts(" END");
}

}  // namespace

extern "C" empi_status empi_run_config(const char* config_path, const empi_engine_opts* opts) {
    if (!config_path) return empi::fail(EMPI_ERR_INVALID_ARGUMENT, "invalidArgument");
    try {
        run_config(config_path, opts);
    } catch (const Error& e) {
        return empi::fail(e.status, e.what());
    } catch (const std::bad_alloc&) {
        return empi::fail(EMPI_ERR_OUT_OF_MEMORY, "insufficientMemory");
    } catch (...) {
        return empi::fail(EMPI_ERR_INTERNAL, "internalError");
    }
    return empi::ok();
}

extern "C" empi_status empi_book_write(const char* path, int append, int epoch_number, double fs, int channels,
                                       int n, const float* samples, int cap, const double* atoms,
                                       const int* counts) {
    if (!path || channels <= 0 || n < 0 || (n > 0 && !samples) || !counts)
        return empi::fail(EMPI_ERR_INVALID_ARGUMENT, "invalidArgument");
    try {
        std::vector<uint8_t> b;
        if (!append) book_header(b, channels, fs);
        book_epoch(b, epoch_number, channels, n, samples, cap, atoms, counts);
        write_file(path, b, append != 0);
    } catch (const Error& e) {
        return empi::fail(e.status, e.what());
    }
    return empi::ok();
}
