// api_tool.cpp — exercises the reference-shaped C++ API (swiftimpute/imputer.hpp)
// the way a caller of the reference would: load VCFs, build the index, impute,
// write the VCF. Used by tests/test_cpp_api.py.
//
//   api_tool parse  <ref.vcf> <tgt.vcf> <prefix>     (no GPU) dump panel / GL, binary round trip
//   api_tool impute <ref.vcf> <tgt.vcf> <out.vcf> <prefix> <deterministic> <L> <ne> [posteriors]
#include "swiftimpute/imputer.hpp"

#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>

using namespace swiftimpute;

static void dump(const std::string& path, const void* p, size_t n) {
    std::ofstream o(path, std::ios::binary);
    o.write(static_cast<const char*>(p), n);
}

int main(int argc, char** argv) {
    if (argc < 5) return 2;
    const std::string cmd = argv[1];
    try {
        auto ref = ReferencePanel::load_vcf(argv[2]);
        auto tgt = TargetData::load_vcf(argv[3]);
        if (cmd == "parse") {
            const std::string pre = argv[4];
            dump(pre + ".panel", ref->haplotypes(), (size_t)ref->num_markers() * ref->num_haplotypes());
            dump(pre + ".gl", tgt->genotype_likelihoods(),
                 (size_t)tgt->num_samples() * tgt->num_markers() * sizeof(GenotypeLikelihoods));
            ref->save_binary(pre + ".sipanel");
            auto back = ReferencePanel::load_binary(pre + ".sipanel");
            const bool same = back->num_markers() == ref->num_markers() &&
                              back->num_haplotypes() == ref->num_haplotypes() &&
                              std::memcmp(back->haplotypes(), ref->haplotypes(),
                                          (size_t)ref->num_markers() * ref->num_haplotypes()) == 0 &&
                              back->markers()[1].pos == ref->markers()[1].pos &&
                              back->markers()[1].id == ref->markers()[1].id;
            // a result written without a device: phased alleles from the panel's first two haplotypes
            ImputationResult r(tgt->num_samples(), tgt->num_markers());
            std::vector<allele_t> h(tgt->num_markers());
            for (sample_t s = 0; s < tgt->num_samples(); ++s)
                for (uint32_t ph = 0; ph < 2; ++ph) {
                    for (marker_t m = 0; m < tgt->num_markers(); ++m) h[m] = ref->get_allele(m, ph);
                    r.set_haplotype(s, ph, h.data());
                }
            r.compute_info_scores();
            ImputationConfig cfg;
            r.write_vcf(pre + ".out.vcf", *tgt, *ref, cfg);
            std::printf("M=%u N=%u B=%u roundtrip=%d info0=%.4f\n", ref->num_markers(), ref->num_haplotypes(),
                        tgt->num_samples(), same ? 1 : 0, r.get_info_score(0));
            return same ? 0 : 3;
        }
        if (cmd == "impute") {
            ImputationConfig cfg;
            cfg.deterministic = std::atoi(argv[6]) != 0;
            cfg.hmm_params.num_states = (uint32_t)std::atoi(argv[7]);
            cfg.hmm_params.ne = (uint32_t)std::atoi(argv[8]);
            cfg.write_posteriors = argc > 9 && std::atoi(argv[9]) != 0;
            cfg.max_samples_per_call = 7;  // three device passes: results must not depend on it
            Imputer imp(*ref, cfg);
            imp.build_index();
            uint32_t calls = 0, last_done = 0, last_total = 0;
            auto res = imp.impute_with_progress(*tgt, [&](uint32_t done, uint32_t total) {
                ++calls;
                last_done = done;
                last_total = total;
            });
            res->write_vcf(argv[4], *tgt, *ref, cfg);
            const std::string pre = argv[5];
            const size_t n = (size_t)res->num_samples() * res->num_markers();
            dump(pre + ".haps", res->haplotype0(0), 2 * n);
            std::vector<float> ds(n), gp(3 * n), dsh(n);
            for (sample_t s = 0; s < res->num_samples(); ++s)
                for (marker_t m = 0; m < res->num_markers(); ++m) {
                    ds[(size_t)s * res->num_markers() + m] = res->get_posterior_dosage(s, m);
                    dsh[(size_t)s * res->num_markers() + m] = res->get_dosage(s, m);
                    res->get_probabilities(s, m, &gp[3 * ((size_t)s * res->num_markers() + m)]);
                }
            dump(pre + ".dosage", ds.data(), n * 4);
            dump(pre + ".hard", dsh.data(), n * 4);
            dump(pre + ".gp", gp.data(), 3 * n * 4);
            std::printf("impute ok: B=%u M=%u progress_calls=%u last=%u/%u device_bytes=%zu\n", res->num_samples(),
                        res->num_markers(), calls, last_done, last_total, imp.device_memory_usage());
            return 0;
        }
    } catch (const CUDAError& e) {
        std::printf("CUDAError: %s\n", e.what());
        return 10;
    } catch (const ImputationError& e) {
        std::printf("ImputationError: %s\n", e.what());
        return 11;
    } catch (const std::exception& e) {
        std::printf("error: %s\n", e.what());
        return 12;
    }
    return 2;
}
