// host_api.cpp — the reference's C++ API (include/swiftimpute/imputer.hpp)
// implemented over the C ABI. VCF parsing/writing stays on the host and keeps
// the reference's text conventions (src/io/vcf_reader.hpp:420-562,
// src/io/vcf_writer.hpp:99-250) so files round-trip the same way.
#include "../../include/swiftimpute/imputer.hpp"
#include "../../include/swiftimpute_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <exception>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <mutex>
#include <sstream>
#include <thread>

namespace swiftimpute {
namespace {

constexpr prob_t kLog10Zero = -999.0f;  // imputer.cpp:244

struct VcfVariant {
    std::string chrom, id, ref;
    uint64_t pos = 0;
    std::vector<std::string> alt;
    std::vector<std::vector<allele_t>> gts;
};

struct VcfFile {
    std::vector<std::string> samples;
    std::vector<std::string> contigs;
    std::vector<VcfVariant> variants;
};

// GT subfield: text before the first ':'; "a|b" / "a/b" diploid, else haploid;
// "." is missing (vcf_reader.hpp:534-562).
std::vector<allele_t> parse_gt(const std::string& cell) {
    std::vector<allele_t> gt;
    const std::string f = cell.substr(0, cell.find(':'));
    const size_t d = f.find_first_of("|/");
    auto one = [](const std::string& a) -> allele_t {
        if (a == "." || a.empty()) return ALLELE_MISSING;
        return static_cast<allele_t>(std::stoi(a));
    };
    if (d == std::string::npos) {
        gt.push_back(one(f));
    } else {
        gt.push_back(one(f.substr(0, d)));
        gt.push_back(one(f.substr(d + 1)));
    }
    return gt;
}

// "chrom", "chrom:start-end" (1-based, inclusive) or "" (everything).
bool in_region(const std::string& region, const std::string& chrom, uint64_t pos) {
    if (region.empty()) return true;
    const size_t c = region.find(':');
    if (c == std::string::npos) return chrom == region;
    if (chrom != region.substr(0, c)) return false;
    std::string span = region.substr(c + 1);
    span.erase(std::remove(span.begin(), span.end(), ','), span.end());
    const size_t dash = span.find('-');
    const uint64_t lo = std::stoull(span.substr(0, dash));
    const uint64_t hi = dash == std::string::npos ? UINT64_MAX : std::stoull(span.substr(dash + 1));
    return pos >= lo && pos <= hi;
}

VcfFile read_vcf(const std::string& filename, const std::string& region) {
    std::ifstream in(filename);
    if (!in) throw std::runtime_error("Cannot open VCF file: " + filename);
    if (filename.size() > 3 && filename.compare(filename.size() - 3, 3, ".gz") == 0)
        throw std::runtime_error("Compressed VCF input is not supported by the plain-text reader: " + filename);
    VcfFile v;
    std::string line;
    while (std::getline(in, line)) {
        if (line.empty()) continue;
        if (line.rfind("##", 0) == 0) {
            if (line.rfind("##contig=", 0) == 0) {
                size_t a = line.find("ID=");
                if (a != std::string::npos) {
                    a += 3;
                    const size_t b = line.find_first_of(",>", a);
                    if (b != std::string::npos) v.contigs.push_back(line.substr(a, b - a));
                }
            }
            continue;
        }
        if (line[0] == '#') {
            std::istringstream iss(line);
            std::vector<std::string> cols;
            std::string c;
            while (iss >> c) cols.push_back(c);
            if (cols.size() > 9) v.samples.assign(cols.begin() + 9, cols.end());
            continue;
        }
        std::vector<std::string> f;
        {
            std::string x;
            std::istringstream iss(line);
            while (std::getline(iss, x, '\t')) f.push_back(x);
        }
        if (f.size() < 9) continue;
        VcfVariant var;
        var.chrom = f[0];
        var.pos = std::stoull(f[1]);
        if (!in_region(region, var.chrom, var.pos)) continue;
        var.id = f[2];
        var.ref = f[3];
        std::istringstream alts(f[4]);
        std::string a;
        while (std::getline(alts, a, ',')) var.alt.push_back(a);
        for (size_t i = 9; i < f.size(); ++i) var.gts.push_back(parse_gt(f[i]));
        v.variants.push_back(std::move(var));
    }
    return v;
}

std::vector<Marker> to_markers(const VcfFile& v) {
    std::vector<Marker> ms;
    ms.reserve(v.variants.size());
    for (const auto& var : v.variants) {
        Marker m;
        m.chrom = var.chrom;
        m.pos = var.pos;
        m.id = var.id;
        m.ref = var.ref;
        m.alt = var.alt.empty() ? "" : var.alt[0];
        m.cM = 0.0;  // the reference reads no genetic map (imputer.cpp:65)
        ms.push_back(std::move(m));
    }
    return ms;
}

std::vector<Sample> to_samples(const std::vector<std::string>& names) {
    std::vector<Sample> s;
    for (size_t i = 0; i < names.size(); ++i) {
        Sample x(names[i]);
        x.index = static_cast<uint32_t>(i);
        s.push_back(std::move(x));
    }
    return s;
}

GenotypeLikelihoods hard_call_gl(allele_t a, allele_t b, bool present) {
    GenotypeLikelihoods g;  // missing = {0,0,0}
    if (!present || a == ALLELE_MISSING || b == ALLELE_MISSING) return g;
    if (a == 0 && b == 0) { g.ll_01 = kLog10Zero; g.ll_11 = kLog10Zero; }
    else if ((a == 0 && b == 1) || (a == 1 && b == 0)) { g.ll_00 = kLog10Zero; g.ll_11 = kLog10Zero; }
    else if (a == 1 && b == 1) { g.ll_00 = kLog10Zero; g.ll_01 = kLog10Zero; }
    return g;
}

std::string fmt4(double x) {
    std::ostringstream o;
    o << std::fixed << std::setprecision(4) << x;
    return o.str();
}

}  // namespace

// ---------------------------------------------------------------- Logger, devices

Logger& Logger::instance() {
    static Logger logger;
    return logger;
}

void Logger::log(Level level, const std::string& prefix, const std::string& msg) {
    if (level < level_) return;
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    std::cout << prefix << msg << std::endl;
}
void Logger::debug(const std::string& msg) { log(DEBUG, "[DEBUG] ", msg); }
void Logger::info(const std::string& msg) { log(INFO, "[INFO] ", msg); }
void Logger::warning(const std::string& msg) { log(WARNING, "[WARNING] ", msg); }
void Logger::error(const std::string& msg) { log(ERROR, "[ERROR] ", msg); }

DeviceInfo get_device_info(int device_id) {
    DeviceInfo info;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device_id) != cudaSuccess) {
        cudaGetLastError();
        throw CUDAError("cudaGetDeviceProperties", 100);
    }
    info.device_id = device_id;
    info.name = prop.name;
    info.total_memory = prop.totalGlobalMem;
    info.compute_capability_major = prop.major;
    info.compute_capability_minor = prop.minor;
    info.multiprocessor_count = prop.multiProcessorCount;
    info.max_threads_per_block = prop.maxThreadsPerBlock;
    info.max_threads_per_multiprocessor = prop.maxThreadsPerMultiProcessor;
    int cur = 0;
    cudaGetDevice(&cur);
    if (cudaSetDevice(device_id) == cudaSuccess) {
        size_t f = 0, t = 0;
        if (cudaMemGetInfo(&f, &t) == cudaSuccess) info.free_memory = f;
        cudaSetDevice(cur);
    }
    return info;
}

int select_best_device() {  // most free memory (types.cpp:69-90)
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        throw CUDAError("no CUDA device", 100);
    }
    int best = 0;
    size_t best_free = 0;
    for (int d = 0; d < n; ++d) {
        const size_t f = get_available_gpu_memory(d);
        if (f > best_free) { best_free = f; best = d; }
    }
    return best;
}

size_t get_available_gpu_memory(int device_id) {
    int cur = 0;
    cudaGetDevice(&cur);
    size_t f = 0, t = 0;
    if (cudaSetDevice(device_id) == cudaSuccess && cudaMemGetInfo(&f, &t) == cudaSuccess) {
        cudaSetDevice(cur);
        return f;
    }
    cudaGetLastError();
    return 0;
}

size_t get_total_gpu_memory(int device_id) {
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device_id) != cudaSuccess) { cudaGetLastError(); return 0; }
    return prop.totalGlobalMem;
}

// ---------------------------------------------------------------- ReferencePanel

std::unique_ptr<ReferencePanel> ReferencePanel::load_vcf(const std::string& filename, const std::string& region) {
    VcfFile v = read_vcf(filename, region);
    if (v.variants.empty()) throw ImputationError("No variants found in reference VCF");
    const haplotype_t N = static_cast<haplotype_t>(v.samples.size() * 2);
    const size_t M = v.variants.size();
    auto h = std::make_unique<allele_t[]>(M * N);
    for (size_t m = 0; m < M; ++m) {  // imputer.cpp:85-112
        for (size_t s = 0; s < v.samples.size(); ++s) {
            allele_t a = ALLELE_MISSING, b = ALLELE_MISSING;
            if (s < v.variants[m].gts.size()) {
                const auto& gt = v.variants[m].gts[s];
                if (gt.size() >= 2) { a = gt[0]; b = gt[1]; }
                else if (gt.size() == 1) { a = gt[0]; b = gt[0]; }
            }
            h[m * N + 2 * s] = a;
            h[m * N + 2 * s + 1] = b;
        }
    }
    return from_haplotypes(to_markers(v), to_samples(v.samples), N, std::move(h));
}

std::unique_ptr<ReferencePanel> ReferencePanel::from_haplotypes(std::vector<Marker> markers,
                                                                std::vector<Sample> samples,
                                                                haplotype_t num_haplotypes,
                                                                std::unique_ptr<allele_t[]> haplotypes) {
    auto p = std::make_unique<ReferencePanel>();
    p->markers_ = std::move(markers);
    p->samples_ = std::move(samples);
    p->num_haplotypes_ = num_haplotypes;
    p->haplotypes_ = std::move(haplotypes);
    return p;
}

namespace {

void put_u32(std::ostream& o, uint32_t x) { o.write(reinterpret_cast<const char*>(&x), 4); }
void put_str(std::ostream& o, const std::string& s) {
    put_u32(o, (uint32_t)s.size());
    o.write(s.data(), s.size());
}
uint32_t get_u32(std::istream& in) {
    uint32_t x = 0;
    in.read(reinterpret_cast<char*>(&x), 4);
    return x;
}
std::string get_str(std::istream& in) {
    const uint32_t n = get_u32(in);
    if (!in) throw ImputationError("truncated binary file header");
    if (n > (1u << 20)) throw ImputationError("corrupt string field in binary file");
    std::string s(n, '\0');
    in.read(&s[0], n);
    return s;
}

// per marker: chrom, id, ref, alt (u32 length + bytes), pos (u64), cM (f64);
// then the sample count and ids. The same in panel and target files.
void put_meta(std::ostream& o, const std::vector<Marker>& markers, const std::vector<Sample>& samples) {
    for (const auto& m : markers) {
        put_str(o, m.chrom); put_str(o, m.id); put_str(o, m.ref); put_str(o, m.alt);
        o.write(reinterpret_cast<const char*>(&m.pos), 8);
        o.write(reinterpret_cast<const char*>(&m.cM), 8);
    }
    put_u32(o, (uint32_t)samples.size());
    for (const auto& s : samples) put_str(o, s.id);
}
void get_meta(std::istream& in, uint32_t M, std::vector<Marker>& markers, std::vector<std::string>& names) {
    if (!in) throw ImputationError("truncated binary file header");
    // grown entry by entry: a damaged count fails at the end of the file, not in one huge allocation
    markers.clear();
    markers.reserve(std::min<uint32_t>(M, 1u << 16));
    for (uint32_t i = 0; i < M; ++i) {
        Marker m;
        m.chrom = get_str(in); m.id = get_str(in); m.ref = get_str(in); m.alt = get_str(in);
        in.read(reinterpret_cast<char*>(&m.pos), 8);
        in.read(reinterpret_cast<char*>(&m.cM), 8);
        markers.push_back(std::move(m));
    }
    const uint32_t n_names = get_u32(in);
    names.clear();
    names.reserve(std::min<uint32_t>(n_names, 1u << 16));
    for (uint32_t i = 0; i < n_names && in; ++i) names.push_back(get_str(in));
    if (!in) throw ImputationError("truncated binary file header");
}

// the body that follows the header must be there before it is allocated
void check_body(std::istream& in, uint64_t rows, uint64_t row_bytes, const char* what, const std::string& filename) {
    const std::streampos here = in.tellg();
    in.seekg(0, std::ios::end);
    const std::streampos end = in.tellg();
    in.seekg(here);
    if (here < 0 || end < here || (uint64_t)(end - here) < rows * row_bytes)
        throw ImputationError(std::string("truncated ") + what + ": " + filename);
}

void check_magic(std::istream& in, const char* magic, const char* what, const std::string& filename) {
    char got[8];
    in.read(got, 8);
    if (!in || std::memcmp(got, magic, 8) != 0) throw ImputationError(std::string("not a ") + what + ": " + filename);
}

}  // namespace

// Binary panel: magic "SIPANEL1", M and N (u32), the markers and sample ids,
// then the alleles bit-packed per marker: ceil(N/8) bytes, haplotype h at bit
// h%8 of byte h/8 (bit set for a non-zero allele). A panel with alleles other
// than 0 and 1 (ALLELE_MISSING, multi-allelic indices) is written as
// "SIPANEL2": the same, followed by their count (u64) and, in marker then
// haplotype order, each as marker (u32), haplotype (u32) and byte (u8).
void ReferencePanel::save_binary(const std::string& filename) const {
    std::ofstream o(filename, std::ios::binary);
    if (!o) throw ImputationError("Cannot write " + filename);
    const size_t cells = (size_t)num_markers() * num_haplotypes_;
    uint64_t n_other = 0;
    for (size_t i = 0; i < cells; ++i) n_other += haplotypes_[i] > 1;
    o.write(n_other ? "SIPANEL2" : "SIPANEL1", 8);
    put_u32(o, num_markers());
    put_u32(o, num_haplotypes_);
    put_meta(o, markers_, samples_);
    const size_t rb = (num_haplotypes_ + 7) / 8;
    std::vector<char> row(rb);
    for (marker_t m = 0; m < num_markers(); ++m) {
        std::fill(row.begin(), row.end(), 0);
        for (haplotype_t h = 0; h < num_haplotypes_; ++h)
            if (haplotypes_[(size_t)m * num_haplotypes_ + h]) row[h / 8] |= (char)(1u << (h % 8));
        o.write(row.data(), rb);
    }
    if (n_other) {
        o.write(reinterpret_cast<const char*>(&n_other), 8);
        for (marker_t m = 0; m < num_markers(); ++m)
            for (haplotype_t h = 0; h < num_haplotypes_; ++h) {
                const allele_t a = haplotypes_[(size_t)m * num_haplotypes_ + h];
                if (a <= 1) continue;
                put_u32(o, m);
                put_u32(o, h);
                o.write(reinterpret_cast<const char*>(&a), 1);
            }
    }
    if (!o) throw ImputationError("write failed: " + filename);
}

std::unique_ptr<ReferencePanel> ReferencePanel::load_binary(const std::string& filename) {
    std::ifstream in(filename, std::ios::binary);
    if (!in) throw ImputationError("Cannot open " + filename);
    char magic[8];
    in.read(magic, 8);
    const bool v1 = in && std::memcmp(magic, "SIPANEL1", 8) == 0, v2 = in && std::memcmp(magic, "SIPANEL2", 8) == 0;
    if (!v1 && !v2) throw ImputationError("not a binary panel: " + filename);
    const uint32_t M = get_u32(in), N = get_u32(in);
    std::vector<Marker> ms;
    std::vector<std::string> names;
    get_meta(in, M, ms, names);
    const size_t rb = (N + 7) / 8;
    check_body(in, M, rb, "binary panel", filename);
    auto h = std::make_unique<allele_t[]>((size_t)M * N);
    std::vector<unsigned char> row(rb);
    for (uint32_t m = 0; m < M; ++m) {
        in.read(reinterpret_cast<char*>(row.data()), rb);
        for (uint32_t j = 0; j < N; ++j) h[(size_t)m * N + j] = (row[j / 8] >> (j % 8)) & 1u;
    }
    if (!in) throw ImputationError("truncated binary panel: " + filename);
    if (v2) {
        uint64_t n_other = 0;
        in.read(reinterpret_cast<char*>(&n_other), 8);
        check_body(in, n_other, 9, "binary panel", filename);
        for (uint64_t i = 0; i < n_other && in; ++i) {
            const uint32_t m = get_u32(in), j = get_u32(in);
            unsigned char a = 0;
            in.read(reinterpret_cast<char*>(&a), 1);
            if (!in) break;
            if (m >= M || j >= N || a <= 1 || !h[(size_t)m * N + j])
                throw ImputationError("corrupt allele entry in binary panel: " + filename);
            h[(size_t)m * N + j] = a;
        }
        if (!in) throw ImputationError("truncated binary panel: " + filename);
    }
    return from_haplotypes(std::move(ms), to_samples(names), N, std::move(h));
}

allele_t ReferencePanel::get_allele(marker_t m, haplotype_t h) const {
    if (m >= markers_.size() || h >= num_haplotypes_) return ALLELE_MISSING;
    return haplotypes_[(size_t)m * num_haplotypes_ + h];
}

size_t ReferencePanel::memory_usage() const {
    size_t t = markers_.capacity() * sizeof(Marker) + samples_.capacity() * sizeof(Sample);
    return t + (size_t)markers_.size() * num_haplotypes_;
}

// ---------------------------------------------------------------- TargetData

std::unique_ptr<TargetData> TargetData::load_vcf(const std::string& filename, const std::string& region) {
    VcfFile v = read_vcf(filename, region);
    if (v.variants.empty()) throw ImputationError("No variants found in target VCF");
    auto t = std::make_unique<TargetData>();
    t->markers_ = to_markers(v);
    t->samples_ = to_samples(v.samples);
    const size_t M = v.variants.size(), B = v.samples.size();
    t->genotype_liks_ = std::make_unique<GenotypeLikelihoods[]>(B * M);
    for (size_t m = 0; m < M; ++m)  // imputer.cpp:247-296
        for (size_t s = 0; s < B; ++s) {
            const bool present = s < v.variants[m].gts.size() && v.variants[m].gts[s].size() >= 2;
            const auto& gt = v.variants[m].gts.size() > s ? v.variants[m].gts[s] : std::vector<allele_t>();
            t->genotype_liks_[s * M + m] = present ? hard_call_gl(gt[0], gt[1], true) : GenotypeLikelihoods();
        }
    return t;
}

std::unique_ptr<TargetData> TargetData::from_genotypes(std::vector<Marker> markers, std::vector<Sample> samples,
                                                       const uint8_t* codes) {
    auto t = std::make_unique<TargetData>();
    const size_t M = markers.size(), B = samples.size();
    t->markers_ = std::move(markers);
    t->samples_ = std::move(samples);
    t->genotype_liks_ = std::make_unique<GenotypeLikelihoods[]>(B * M);
    for (size_t i = 0; i < B * M; ++i) {
        const uint8_t c = codes[i];
        t->genotype_liks_[i] = c == 0 ? hard_call_gl(0, 0, true)
                               : c == 1 ? hard_call_gl(0, 1, true)
                               : c == 2 ? hard_call_gl(1, 1, true)
                                        : GenotypeLikelihoods();
    }
    return t;
}

namespace {

// the four likelihood triples a target cell can hold (imputer.cpp:263-287)
// and their genotype codes: 0/1/2 ALT alleles, 3 = missing
uint8_t gl_code(const GenotypeLikelihoods& g) {
    const auto is = [&](prob_t a, prob_t b, prob_t c) { return g.ll_00 == a && g.ll_01 == b && g.ll_11 == c; };
    if (is(0.f, kLog10Zero, kLog10Zero)) return 0;
    if (is(kLog10Zero, 0.f, kLog10Zero)) return 1;
    if (is(kLog10Zero, kLog10Zero, 0.f)) return 2;
    if (g.ll_00 == g.ll_01 && g.ll_01 == g.ll_11) return 3;
    throw ImputationError("binary target format stores hard calls and missing cells only");
}

}  // namespace

// Binary targets: magic "SITARGT1", M (u32), the markers and sample ids, then
// one row of ceil(M/4) bytes per sample, the code of marker m at bits
// 2(m%4)..2(m%4)+1 of byte m/4: 2 bits per cell instead of the 12-byte
// likelihood triple
void TargetData::save_binary(const std::string& filename) const {
    std::ofstream o(filename, std::ios::binary);
    if (!o) throw ImputationError("Cannot write " + filename);
    o.write("SITARGT1", 8);
    put_u32(o, (uint32_t)markers_.size());
    put_meta(o, markers_, samples_);
    const size_t M = markers_.size(), rb = (M + 3) / 4;
    std::vector<unsigned char> row(rb);
    for (size_t s = 0; s < samples_.size(); ++s) {
        std::fill(row.begin(), row.end(), 0);
        for (size_t m = 0; m < M; ++m) row[m / 4] |= (unsigned char)(gl_code(genotype_liks_[s * M + m]) << (2 * (m % 4)));
        o.write(reinterpret_cast<const char*>(row.data()), rb);
    }
    if (!o) throw ImputationError("write failed: " + filename);
}

std::unique_ptr<TargetData> TargetData::load_binary(const std::string& filename) {
    std::ifstream in(filename, std::ios::binary);
    if (!in) throw ImputationError("Cannot open " + filename);
    check_magic(in, "SITARGT1", "binary target file", filename);
    const uint32_t n_markers = get_u32(in);
    std::vector<Marker> ms;
    std::vector<std::string> names;
    get_meta(in, n_markers, ms, names);
    const size_t M = ms.size(), B = names.size(), rb = (M + 3) / 4;
    check_body(in, B, rb, "binary target file", filename);
    std::vector<uint8_t> codes(B * M);
    std::vector<unsigned char> row(rb);
    for (size_t s = 0; s < B; ++s) {
        in.read(reinterpret_cast<char*>(row.data()), rb);
        for (size_t m = 0; m < M; ++m) codes[s * M + m] = (row[m / 4] >> (2 * (m % 4))) & 3u;
    }
    if (!in) throw ImputationError("truncated binary target file: " + filename);
    return from_genotypes(std::move(ms), to_samples(names), codes.data());
}

GenotypeLikelihoods TargetData::get_likelihood(sample_t s, marker_t m) const {
    if (s >= samples_.size() || m >= markers_.size()) return GenotypeLikelihoods();
    return genotype_liks_[(size_t)s * markers_.size() + m];
}

size_t TargetData::memory_usage() const {
    return markers_.capacity() * sizeof(Marker) + samples_.capacity() * sizeof(Sample) +
           samples_.size() * markers_.size() * sizeof(GenotypeLikelihoods);
}

// ---------------------------------------------------------------- ImputationResult

ImputationResult::ImputationResult(uint32_t num_samples, uint32_t num_markers)
    : num_samples_(num_samples), num_markers_(num_markers) {
    const size_t n = (size_t)num_samples * num_markers;
    haplotypes_ = std::make_unique<allele_t[]>(2 * n);
    posteriors_ = std::make_unique<prob_t[]>(2 * n);
    dosages_ = std::make_unique<prob_t[]>(n);
    info_scores_ = std::make_unique<prob_t[]>(num_markers);
    std::fill(haplotypes_.get(), haplotypes_.get() + 2 * n, 0);
    std::fill(posteriors_.get(), posteriors_.get() + 2 * n, 0.0f);
    std::fill(dosages_.get(), dosages_.get() + n, 0.0f);
    std::fill(info_scores_.get(), info_scores_.get() + num_markers, 0.0f);
}

const allele_t* ImputationResult::haplotype0(sample_t s) const {
    return s < num_samples_ ? &haplotypes_[(size_t)s * 2 * num_markers_] : nullptr;
}
const allele_t* ImputationResult::haplotype1(sample_t s) const {
    return s < num_samples_ ? &haplotypes_[(size_t)s * 2 * num_markers_ + num_markers_] : nullptr;
}

prob_t ImputationResult::get_dosage(sample_t s, marker_t m) const {
    if (s >= num_samples_ || m >= num_markers_) return 0.0f;
    return (prob_t)(haplotypes_[(size_t)s * 2 * num_markers_ + m] +
                    haplotypes_[(size_t)s * 2 * num_markers_ + num_markers_ + m]);
}

prob_t ImputationResult::get_posterior_dosage(sample_t s, marker_t m) const {
    if (s >= num_samples_ || m >= num_markers_) return 0.0f;
    return dosages_[(size_t)s * num_markers_ + m];
}

void ImputationResult::get_probabilities(sample_t s, marker_t m, prob_t probs[3]) const {
    if (s >= num_samples_ || m >= num_markers_) { probs[0] = probs[1] = probs[2] = 0.0f; return; }
    const size_t i = ((size_t)s * num_markers_ + m) * 2;  // imputer.cpp:427-445
    const prob_t p1 = posteriors_[i], q1 = posteriors_[i + 1];
    const prob_t p0 = 1.0f - p1, q0 = 1.0f - q1;
    probs[0] = p0 * q0;
    probs[1] = p0 * q1 + p1 * q0;
    probs[2] = p1 * q1;
}

prob_t ImputationResult::get_info_score(marker_t m) const { return m < num_markers_ ? info_scores_[m] : 0.0f; }

void ImputationResult::set_haplotype(sample_t s, uint32_t phase, const allele_t* h) {
    if (s >= num_samples_ || phase >= 2) return;
    std::copy(h, h + num_markers_, &haplotypes_[(size_t)s * 2 * num_markers_ + (size_t)phase * num_markers_]);
}

void ImputationResult::set_posterior(sample_t s, marker_t m, const prob_t* p) {
    if (s >= num_samples_ || m >= num_markers_) return;
    const size_t i = ((size_t)s * num_markers_ + m) * 2;
    posteriors_[i] = p[0];
    posteriors_[i + 1] = p[1];
}

void ImputationResult::set_posterior_dosage(sample_t s, marker_t m, prob_t d) {
    if (s < num_samples_ && m < num_markers_) dosages_[(size_t)s * num_markers_ + m] = d;
}

// INFO = 1 - Var(dosage) / (2p(1-p)) over the phased-allele dosages (imputer.cpp:467-496)
void ImputationResult::compute_info_scores() {
    for (marker_t m = 0; m < num_markers_; ++m) {
        double sum = 0.0, sq = 0.0;
        for (sample_t s = 0; s < num_samples_; ++s) {
            const double d = get_dosage(s, m);
            sum += d;
            sq += d * d;
        }
        const double mean = sum / num_samples_;
        const double p = mean / 2.0;
        if (p == 0.0 || p == 1.0) { info_scores_[m] = 1.0f; continue; }
        const double var = sq / num_samples_ - mean * mean;
        const double info = 1.0 - var / (2.0 * p * (1.0 - p));
        info_scores_[m] = (prob_t)std::max(0.0, std::min(1.0, info));
    }
}

size_t ImputationResult::memory_usage() const {
    const size_t n = (size_t)num_samples_ * num_markers_;
    return 2 * n + 2 * n * sizeof(prob_t) + n * sizeof(prob_t) + num_markers_ * sizeof(prob_t);
}

// VCF 4.2 with the reference writer's header and GT-only phased rows
// (vcf_writer.hpp:99-132, 212-250); GT:DS:GP rows when write_posteriors is set.
void ImputationResult::write_vcf(const std::string& filename, const TargetData& targets,
                                 const ReferencePanel& reference, const ImputationConfig& config) const {
    std::ofstream o(filename);
    if (!o) throw std::runtime_error("Cannot open file for writing: " + filename);
    if (filename.size() > 3 && filename.compare(filename.size() - 3, 3, ".gz") == 0)
        throw std::runtime_error("Compressed VCF output is not supported: " + filename);
    o << "##fileformat=VCFv4.2\n##source=SwiftImpute\n";
    if (!reference.markers().empty()) o << "##contig=<ID=" << reference.markers()[0].chrom << ">\n";
    o << "##INFO=<ID=IMP,Number=0,Type=Flag,Description=\"Imputed variant\">\n"
      << "##FORMAT=<ID=GT,Number=1,Type=String,Description=\"Genotype\">\n"
      << "##FORMAT=<ID=DS,Number=1,Type=Float,Description=\"Dosage (expected ALT allele count)\">\n"
      << "##FORMAT=<ID=GP,Number=G,Type=Float,Description=\"Genotype posterior probabilities\">\n"
      << "##FORMAT=<ID=AP,Number=2,Type=Float,Description=\"Allelic probabilities\">\n"
      << "#CHROM\tPOS\tID\tREF\tALT\tQUAL\tFILTER\tINFO\tFORMAT";
    for (const auto& s : targets.samples()) o << "\t" << s.id;
    o << "\n";
    for (marker_t m = 0; m < num_markers_; ++m) {
        const Marker& mk = reference.markers()[m];
        o << mk.chrom << "\t" << mk.pos << "\t" << (mk.id.empty() ? "." : mk.id) << "\t" << mk.ref << "\t" << mk.alt
          << "\t.\tPASS\tIMP\t" << (config.write_posteriors ? "GT:DS:GP" : "GT");
        for (sample_t s = 0; s < num_samples_; ++s) {
            const int a = haplotypes_[(size_t)s * 2 * num_markers_ + m];
            const int b = haplotypes_[(size_t)s * 2 * num_markers_ + num_markers_ + m];
            o << "\t" << a << "|" << b;
            if (config.write_posteriors) {
                prob_t gp[3];
                get_probabilities(s, m, gp);
                o << ":" << fmt4(get_posterior_dosage(s, m)) << ":" << fmt4(gp[0]) << "," << fmt4(gp[1]) << ","
                  << fmt4(gp[2]);
            }
        }
        o << "\n";
    }
    if (!o) throw std::runtime_error("write failed: " + filename);
}

// ---------------------------------------------------------------- Imputer

Imputer::Imputer(const ReferencePanel& reference, const ImputationConfig& config)
    : reference_(reference), config_(config) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        throw CUDAError("no CUDA device", 100);
    }
    device_id_ = config_.device_id < 0 ? select_best_device() : config_.device_id;
    check(si_ctx_create(device_id_, config_.hbm_budget_bytes, &ctx_), "si_ctx_create");
}

Imputer::~Imputer() {
    if (ctx_) si_ctx_destroy(ctx_);
}

void Imputer::check(int status, const char* what) const {
    if (status == SI_OK) return;
    std::string msg = std::string(what) + ": " + si_status_string((si_status)status);
    if (ctx_) msg += std::string(" — ") + si_last_error(ctx_);
    if (status == SI_ERR_CUDA || status == SI_ERR_OUT_OF_MEMORY) throw CUDAError(msg, status);
    throw ImputationError(msg);
}

void Imputer::ensure_panel() {
    if (panel_on_device_) return;
    check(si_panel_upload_u8(ctx_, reference_.haplotypes(), reference_.num_markers(), reference_.num_haplotypes()),
          "panel upload");
    std::vector<uint64_t> pos(reference_.num_markers());
    std::vector<double> cm(reference_.num_markers());
    for (marker_t m = 0; m < reference_.num_markers(); ++m) {
        pos[m] = reference_.markers()[m].pos;
        cm[m] = reference_.markers()[m].cM;
    }
    check(si_panel_set_map(ctx_, pos.data(), cm.data()), "genetic map");
    panel_on_device_ = true;
}

void Imputer::build_index() {
    ensure_panel();
    check(si_pbwt_build(ctx_, 0), "PBWT build");
    has_index_ = true;
}

void Imputer::save_index(const std::string& filename) {
    ensure_panel();
    if (!has_index_) throw ImputationError("PBWT index not built");
    uint64_t n = 0;
    check(si_pbwt_stored_bytes(ctx_, &n), "stored index size");
    std::vector<char> buf(n);
    check(si_pbwt_save(ctx_, buf.data(), n), "save index");
    std::ofstream o(filename, std::ios::binary);
    if (!o) throw ImputationError("Cannot write " + filename);
    o.write(buf.data(), (std::streamsize)n);
    if (!o) throw ImputationError("write failed: " + filename);
}

void Imputer::load_index(const std::string& filename) {
    ensure_panel();
    std::ifstream in(filename, std::ios::binary | std::ios::ate);
    if (!in) throw ImputationError("Cannot open " + filename);
    const std::streamoff n = in.tellg();
    if (n <= 0) throw ImputationError("empty index file: " + filename);
    in.seekg(0);
    std::vector<char> buf((size_t)n);
    in.read(buf.data(), n);
    if (!in) throw ImputationError("truncated index file: " + filename);
    check(si_pbwt_load(ctx_, buf.data(), (uint64_t)n), "load index");
    has_index_ = true;
}

std::unique_ptr<ImputationResult> Imputer::impute(const TargetData& targets) {
    return impute_with_progress(targets, nullptr);
}

std::unique_ptr<ImputationResult> Imputer::impute_with_progress(
    const TargetData& targets, std::function<void(uint32_t, uint32_t)> progress_callback) {
    auto result = std::make_unique<ImputationResult>(targets.num_samples(), targets.num_markers());
    impute_rows(targets, 0, targets.num_samples(), *result, progress_callback);
    result->compute_info_scores();
    return result;
}

void Imputer::impute_rows(const TargetData& targets, sample_t begin, sample_t end, ImputationResult& result,
                          const std::function<void(uint32_t, uint32_t)>& progress_callback) {
    if (targets.num_markers() != reference_.num_markers())  // imputer.cpp:730-741
        throw ImputationError("Target and reference marker counts don't match: " +
                              std::to_string(targets.num_markers()) + " vs " +
                              std::to_string(reference_.num_markers()));
    ensure_panel();
    const uint32_t B = end - begin, M = targets.num_markers();
    si_impute_params p;
    si_impute_params_default(&p);
    p.num_states = config_.hmm_params.num_states;
    p.ne = config_.hmm_params.ne;
    p.rho_rate = (double)config_.hmm_params.rho_rate;
    p.theta = (double)config_.hmm_params.theta;
    p.transition_mode = config_.transition_mode;
    // without an index (or with PBWT selection off) the reference takes the
    // first L haplotype pairs (2k, 2k+1) (imputer.cpp:929-942)
    p.selection_kind = (has_index_ && config_.hmm_params.use_pbwt_selection) ? SI_SEL_AUTO : SI_SEL_FIRST_PAIRS;
    p.sampling = config_.deterministic ? SI_SAMPLE_ARGMAX : SI_SAMPLE_PHILOX;
    p.seed = config_.seed;
    p.tie_eps = config_.tie_eps;
    p.checkpoint_interval = config_.checkpoint_interval <= 32 ? config_.checkpoint_interval : 0;
    // results do not depend on the chunking: Philox draws are keyed by the global sample index
    const uint64_t per_sample = (uint64_t)M * (12 + 1 + 4 + 8 + 2) + 64;
    uint64_t used = 0, budget = 0;
    si_ctx_memory(ctx_, &used, &budget);
    const uint64_t room = budget > used ? (budget - used) / 2 : 0;
    uint32_t chunk = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(B, room / per_sample));
    chunk = std::max<uint32_t>(std::min<uint32_t>(chunk, B), std::min<uint32_t>(B, config_.batch_size));
    if (config_.max_samples_per_call) chunk = std::min<uint32_t>(chunk, config_.max_samples_per_call);
    for (uint32_t s0 = begin; s0 < end; s0 += chunk) {
        const uint32_t n = std::min(chunk, end - s0);
        p.sample_id_base = s0;
        check(si_impute_gl(ctx_, &p, reinterpret_cast<const float*>(targets.genotype_likelihoods() + (size_t)s0 * M), n,
                           result.dosage_data() + (size_t)s0 * M, result.posterior_data() + (size_t)s0 * M * 2,
                           result.haplotype_data() + (size_t)s0 * 2 * M),
              "imputation");
        if (progress_callback) progress_callback(s0 + n - begin, B);
    }
}

size_t Imputer::device_memory_usage() const {
    uint64_t used = 0, budget = 0;
    si_ctx_memory(ctx_, &used, &budget);
    return (size_t)used;
}

size_t Imputer::estimate_memory_requirement(const ReferencePanel& reference, uint32_t num_target_samples,
                                            const ImputationConfig& config) {
    const size_t M = reference.num_markers(), N = reference.num_haplotypes();
    const size_t words = ((N + 31) / 32 + 3) & ~size_t(3);
    size_t total = M * words * 4 + M * 128 * 4 + M * 8 * 3;                  // bit panel, head rows, tables
    const size_t L = config.hmm_params.num_states;
    const size_t lmax = L <= 4 ? 4 : L <= 8 ? 8 : L <= 16 ? 16 : 32;
    total += (size_t)num_target_samples * M * (1 + 4 + 8 + 2);               // codes in, dosage/P/haps out
    total += (size_t)num_target_samples * (M / 16 + 1) * lmax * 4;           // forward checkpoints
    return total;
}

// ---------------------------------------------------------------- MultiGPUImputer

MultiGPUImputer::MultiGPUImputer(const ReferencePanel& reference, const std::vector<int>& device_ids,
                                 const ImputationConfig& config)
    : reference_(reference), config_(config), device_ids_(device_ids) {
    if (device_ids_.empty()) throw ImputationError("MultiGPUImputer needs at least one device id");
    std::map<int, uint32_t> replicas_on;
    for (int d : device_ids_) ++replicas_on[d];
    for (int d : device_ids_) {
        if (d < 0) throw ImputationError("device id " + std::to_string(d) + " is negative");
        ImputationConfig c = config_;
        c.device_id = d;
        // replicas that share a device split its free memory, unless the config sets a budget
        if (c.hbm_budget_bytes == 0 && replicas_on[d] > 1) {
            size_t free_b = 0, total_b = 0;
            if (cudaSetDevice(d) == cudaSuccess && cudaMemGetInfo(&free_b, &total_b) == cudaSuccess)
                c.hbm_budget_bytes = free_b / replicas_on[d];
            else
                cudaGetLastError();
        }
        imputers_.push_back(std::make_unique<Imputer>(reference_, c));
    }
}

MultiGPUImputer::~MultiGPUImputer() = default;

namespace {

// runs fn(i) for every replica on its own host thread; the first exception
// (in replica order) is rethrown after all threads have joined
template <class Fn>
void on_every_replica(size_t n, Fn fn) {
    std::vector<std::exception_ptr> errors(n);
    std::vector<std::thread> threads;
    threads.reserve(n);
    for (size_t i = 0; i < n; ++i)
        threads.emplace_back([&, i] {
            try {
                fn(i);
            } catch (...) {
                errors[i] = std::current_exception();
            }
        });
    for (auto& t : threads) t.join();
    for (auto& e : errors)
        if (e) std::rethrow_exception(e);
}

}  // namespace

void MultiGPUImputer::build_indices() {
    on_every_replica(imputers_.size(), [&](size_t i) { imputers_[i]->build_index(); });
}

void MultiGPUImputer::partition_samples(uint32_t num_samples, std::vector<uint32_t>& start_indices,
                                        std::vector<uint32_t>& end_indices) const {
    const uint32_t g = (uint32_t)imputers_.size(), base = num_samples / g, extra = num_samples % g;
    start_indices.clear();
    end_indices.clear();
    uint32_t s = 0;
    for (uint32_t i = 0; i < g; ++i) {
        const uint32_t n = base + (i < extra ? 1 : 0);
        if (n == 0) continue;
        start_indices.push_back(s);
        end_indices.push_back(s + n);
        s += n;
    }
}

std::unique_ptr<ImputationResult> MultiGPUImputer::impute(const TargetData& targets) {
    if (targets.num_markers() != reference_.num_markers())
        throw ImputationError("Target and reference marker counts don't match: " +
                              std::to_string(targets.num_markers()) + " vs " +
                              std::to_string(reference_.num_markers()));
    auto result = std::make_unique<ImputationResult>(targets.num_samples(), targets.num_markers());
    std::vector<uint32_t> starts, ends;
    partition_samples(targets.num_samples(), starts, ends);
    on_every_replica(starts.size(), [&](size_t i) {
        imputers_[i]->impute_rows(targets, starts[i], ends[i], *result, nullptr);
    });
    result->compute_info_scores();
    return result;
}

// ---------------------------------------------------------------- convenience

std::unique_ptr<ImputationResult> impute(const std::string& reference_vcf, const std::string& target_vcf,
                                         const std::string& output_vcf, const ImputationConfig& config) {
    auto reference = ReferencePanel::load_vcf(reference_vcf);
    auto targets = TargetData::load_vcf(target_vcf);
    Imputer imputer(*reference, config);
    imputer.build_index();
    auto result = imputer.impute(*targets);
    result->write_vcf(output_vcf, *targets, *reference, config);
    return result;
}

}  // namespace swiftimpute
