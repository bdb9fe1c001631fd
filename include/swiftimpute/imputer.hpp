// swiftimpute/imputer.hpp — the reference's public C++ API (tcBio/SwiftImpute
// src/api/imputer.hpp:21-295 and src/core/types.hpp:12-90), kept name for name
// so callers drop in; behind it the host code calls the B200 kernels through
// the C ABI in swiftimpute_b200.h. VCF input and output stay on the host.
//
// Differences a caller can see, all deliberate:
//   * ImputationConfig::deterministic is honoured (the reference ignores it and
//     always samples, imputer.cpp:1008-1014): true = argmax slot, false = a
//     Philox draw keyed by (seed, sample index, marker).
//   * ImputationResult carries posterior dosages and P(hap=1): get_probabilities
//     (imputer.cpp:427-445) now reads filled posteriors, and
//     get_posterior_dosage is added. get_dosage keeps the reference meaning
//     (sum of the two phased alleles, imputer.cpp:418-425).
//   * ReferencePanel::from_haplotypes / TargetData::from_genotypes build inputs
//     in memory (the reference's constructors are private, imputer.hpp:98-103,
//     139-143), and load_binary / save_binary work (they throw in the reference);
//     TargetData gains the same pair, storing 2 bits per genotype.
//   * Panel alleles must be 0/1 (the device stores one bit per allele).
#pragma once

#include <cstdint>
#include <functional>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

struct si_ctx;

namespace swiftimpute {

using marker_t = uint32_t;
using sample_t = uint32_t;
using haplotype_t = uint32_t;
using allele_t = uint8_t;
using state_t = uint16_t;
using prob_t = float;

constexpr allele_t ALLELE_MISSING = 255;
constexpr marker_t INVALID_MARKER = 0xFFFFFFFF;
constexpr sample_t INVALID_SAMPLE = 0xFFFFFFFF;

struct Marker {
    std::string chrom;
    uint64_t pos = 0;
    std::string id;
    std::string ref;
    std::string alt;
    double cM = 0.0;
};

struct Sample {
    std::string id;
    uint32_t index = 0;
    Sample() = default;
    explicit Sample(std::string id_) : id(std::move(id_)) {}
};

// log10 genotype likelihoods (core/types.hpp:46-52)
struct GenotypeLikelihoods {
    prob_t ll_00 = 0.0f;
    prob_t ll_01 = 0.0f;
    prob_t ll_11 = 0.0f;
};

// core/types.hpp:77-90
struct HMMParameters {
    prob_t theta = 0.001f;
    prob_t rho_rate = 4.0f;
    uint32_t ne = 10000;
    uint32_t num_states = 8;
    bool use_pbwt_selection = true;
};

// Logger and device queries (core/types.hpp:253-317), used by the reference's CLI.
class Logger {
public:
    enum Level { DEBUG = 0, INFO = 1, WARNING = 2, ERROR = 3 };
    static Logger& instance();
    void set_level(Level level) { level_ = level; }
    Level get_level() const { return level_; }
    void debug(const std::string& msg);
    void info(const std::string& msg);
    void warning(const std::string& msg);
    void error(const std::string& msg);

private:
    Logger() = default;
    Level level_ = INFO;
    void log(Level level, const std::string& prefix, const std::string& msg);
};

#define LOG_DEBUG(msg) ::swiftimpute::Logger::instance().debug(msg)
#define LOG_INFO(msg) ::swiftimpute::Logger::instance().info(msg)
#define LOG_WARNING(msg) ::swiftimpute::Logger::instance().warning(msg)
#define LOG_ERROR(msg) ::swiftimpute::Logger::instance().error(msg)

struct DeviceInfo {
    int device_id = -1;
    std::string name;
    size_t total_memory = 0;
    size_t free_memory = 0;
    int compute_capability_major = 0;
    int compute_capability_minor = 0;
    int multiprocessor_count = 0;
    int max_threads_per_block = 0;
    int max_threads_per_multiprocessor = 0;
};

DeviceInfo get_device_info(int device_id = 0);
int select_best_device();
size_t get_available_gpu_memory(int device_id = 0);
size_t get_total_gpu_memory(int device_id = 0);

class ImputationError : public std::runtime_error {
public:
    explicit ImputationError(const std::string& msg) : std::runtime_error(msg) {}
};

class CUDAError : public ImputationError {
public:
    CUDAError(const std::string& msg, int error_code)
        : ImputationError(msg + " (CUDA error: " + std::to_string(error_code) + ")"), error_code_(error_code) {}
    int error_code() const { return error_code_; }

private:
    int error_code_;
};

// imputer.hpp:21-56, plus the engine's own knobs (defaults keep reference behaviour)
struct ImputationConfig {
    HMMParameters hmm_params;
    int device_id = -1;
    uint32_t batch_size = 100;
    uint32_t num_threads = 4;
    bool use_pinned_memory = true;
    bool output_dosages = true;
    bool output_probabilities = true;
    bool output_info_score = true;
    bool deterministic = false;
    uint32_t window_size = 10000;     // accepted; the device forward-backward is exact over the whole chain
    uint32_t window_overlap = 100;    // accepted, unused (as in the reference)
    uint32_t checkpoint_interval = 0; // 0 = engine default

    // engine additions
    int transition_mode = 0;          // 0: first-gap matrix for every gap (reference); 1: per gap
    uint64_t seed = 12345;            // Philox key when deterministic == false
    double tie_eps = 1e-4;            // argmax tolerance
    uint64_t hbm_budget_bytes = 0;    // 0 = all free device memory
    bool write_posteriors = false;    // write_vcf emits GT:DS:GP instead of the reference's GT only
    uint32_t max_samples_per_call = 0; // 0 = as many samples per device pass as the budget allows
};

class ReferencePanel {
public:
    ReferencePanel() = default;
    static std::unique_ptr<ReferencePanel> load_vcf(const std::string& filename, const std::string& region = "");
    static std::unique_ptr<ReferencePanel> load_binary(const std::string& filename);
    void save_binary(const std::string& filename) const;
    static std::unique_ptr<ReferencePanel> from_haplotypes(std::vector<Marker> markers, std::vector<Sample> samples,
                                                           haplotype_t num_haplotypes,
                                                           std::unique_ptr<allele_t[]> haplotypes);

    marker_t num_markers() const { return static_cast<marker_t>(markers_.size()); }
    haplotype_t num_haplotypes() const { return num_haplotypes_; }
    sample_t num_samples() const { return num_haplotypes_ / 2; }
    const std::vector<Marker>& markers() const { return markers_; }
    const std::vector<Sample>& samples() const { return samples_; }
    const allele_t* haplotypes() const { return haplotypes_.get(); }  // [M][N]
    allele_t get_allele(marker_t m, haplotype_t h) const;
    size_t memory_usage() const;

private:
    std::vector<Marker> markers_;
    std::vector<Sample> samples_;
    haplotype_t num_haplotypes_ = 0;
    std::unique_ptr<allele_t[]> haplotypes_;
};

class TargetData {
public:
    TargetData() = default;
    static std::unique_ptr<TargetData> load_vcf(const std::string& filename, const std::string& region = "");
    // genotype codes [B][M]: 0/1/2 ALT count, 3 (or any other value) = missing
    static std::unique_ptr<TargetData> from_genotypes(std::vector<Marker> markers, std::vector<Sample> samples,
                                                      const uint8_t* codes);
    // 2 bits per cell (the ALT count, 3 = missing) instead of the 12-byte likelihood triple
    static std::unique_ptr<TargetData> load_binary(const std::string& filename);
    void save_binary(const std::string& filename) const;

    marker_t num_markers() const { return static_cast<marker_t>(markers_.size()); }
    sample_t num_samples() const { return static_cast<sample_t>(samples_.size()); }
    const std::vector<Marker>& markers() const { return markers_; }
    const std::vector<Sample>& samples() const { return samples_; }
    const GenotypeLikelihoods* genotype_likelihoods() const { return genotype_liks_.get(); }  // [B][M]
    GenotypeLikelihoods get_likelihood(sample_t s, marker_t m) const;
    size_t memory_usage() const;

private:
    std::vector<Marker> markers_;
    std::vector<Sample> samples_;
    std::unique_ptr<GenotypeLikelihoods[]> genotype_liks_;
};

class ImputationResult {
public:
    ImputationResult(uint32_t num_samples, uint32_t num_markers);

    void write_vcf(const std::string& filename, const TargetData& targets, const ReferencePanel& reference,
                   const ImputationConfig& config) const;

    uint32_t num_samples() const { return num_samples_; }
    uint32_t num_markers() const { return num_markers_; }
    const allele_t* haplotype0(sample_t s) const;
    const allele_t* haplotype1(sample_t s) const;
    prob_t get_dosage(sample_t s, marker_t m) const;           // h0 + h1 of the phased alleles
    prob_t get_posterior_dosage(sample_t s, marker_t m) const; // expected ALT count under the posterior
    void get_probabilities(sample_t s, marker_t m, prob_t probs[3]) const;
    prob_t get_info_score(marker_t m) const;

    void set_haplotype(sample_t s, uint32_t phase, const allele_t* haplotype);
    void set_posterior(sample_t s, marker_t m, const prob_t* posterior);
    void set_posterior_dosage(sample_t s, marker_t m, prob_t dosage);
    void compute_info_scores();
    size_t memory_usage() const;

    // raw arrays, for bulk fills: haplotypes [B][2][M], posteriors [B][M][2], dosages [B][M]
    allele_t* haplotype_data() { return haplotypes_.get(); }
    prob_t* posterior_data() { return posteriors_.get(); }
    prob_t* dosage_data() { return dosages_.get(); }

private:
    uint32_t num_samples_;
    uint32_t num_markers_;
    std::unique_ptr<allele_t[]> haplotypes_;
    std::unique_ptr<prob_t[]> posteriors_;
    std::unique_ptr<prob_t[]> dosages_;
    std::unique_ptr<prob_t[]> info_scores_;
};

class Imputer {
public:
    explicit Imputer(const ReferencePanel& reference, const ImputationConfig& config = ImputationConfig());
    ~Imputer();
    Imputer(const Imputer&) = delete;
    Imputer& operator=(const Imputer&) = delete;

    void build_index();
    bool has_index() const { return has_index_; }
    /* Stored index (save_pbwt_index / load_pbwt_index, pbwt_index.hpp:257-258):
     * the built index to a file, or a file's index for this panel instead of
     * build_index(); a file built on another panel is refused. */
    void save_index(const std::string& filename);
    void load_index(const std::string& filename);
    std::unique_ptr<ImputationResult> impute(const TargetData& targets);
    std::unique_ptr<ImputationResult> impute_with_progress(const TargetData& targets,
                                                           std::function<void(uint32_t, uint32_t)> progress_callback);
    const ImputationConfig& config() const { return config_; }
    size_t device_memory_usage() const;
    static size_t estimate_memory_requirement(const ReferencePanel& reference, uint32_t num_target_samples,
                                              const ImputationConfig& config);

private:
    const ReferencePanel& reference_;
    ImputationConfig config_;
    si_ctx* ctx_ = nullptr;
    bool panel_on_device_ = false;
    bool has_index_ = false;
    int device_id_ = 0;

    void ensure_panel();
    void check(int status, const char* what) const;
    // imputes target rows [begin, end) into the same rows of `result`; Philox
    // draws are keyed by the global row index, so a row does not depend on
    // which call, pass or device imputes it
    void impute_rows(const TargetData& targets, sample_t begin, sample_t end, ImputationResult& result,
                     const std::function<void(uint32_t, uint32_t)>& progress_callback);
    friend class MultiGPUImputer;
};

// Sample-sharded replicas on several devices (src/api/imputer.hpp:298-328; the
// reference's impute() runs everything on the first device). Each device holds
// its own panel and index; impute() splits the targets into contiguous shards
// whose sizes differ by at most one and imputes them on one host thread per
// device, with no traffic between devices. Results are bit-identical to one
// Imputer over all targets. A device id may repeat: each entry is one replica.
class MultiGPUImputer {
public:
    MultiGPUImputer(const ReferencePanel& reference, const std::vector<int>& device_ids,
                    const ImputationConfig& config = ImputationConfig());
    ~MultiGPUImputer();

    void build_indices();
    std::unique_ptr<ImputationResult> impute(const TargetData& targets);
    uint32_t num_gpus() const { return static_cast<uint32_t>(imputers_.size()); }

private:
    const ReferencePanel& reference_;
    ImputationConfig config_;
    std::vector<int> device_ids_;
    std::vector<std::unique_ptr<Imputer>> imputers_;

    void partition_samples(uint32_t num_samples, std::vector<uint32_t>& start_indices,
                           std::vector<uint32_t>& end_indices) const;
};

std::unique_ptr<ImputationResult> impute(const std::string& reference_vcf, const std::string& target_vcf,
                                         const std::string& output_vcf,
                                         const ImputationConfig& config = ImputationConfig());

}  // namespace swiftimpute
