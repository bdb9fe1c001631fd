// api_tool.cpp — exercises the reference-shaped C++ API (swiftimpute/imputer.hpp)
// the way a caller of the reference would: load VCFs, build the index, impute,
// write the VCF. Used by tests/test_cpp_api.py.
//
//   api_tool parse  <ref.vcf> <tgt.vcf> <prefix>     (no GPU) dump panel / GL, binary round trips
//   api_tool impute <ref.vcf> <tgt.vcf> <out.vcf> <prefix> <deterministic> <L> <ne> [posteriors]
//   api_tool loadbin <panel|target> <file>           (no GPU) load a binary file, print its shape
//   api_tool index  <ref.vcf> <tgt.vcf> <index file> build, save and reload the PBWT index
//   api_tool multi  <ref.vcf> <tgt.vcf> <devices> <prefix> <deterministic> <L> <ne>
//                   MultiGPUImputer over a comma-separated device list (repeats allowed),
//                   compared with one Imputer over all targets
#include "swiftimpute/imputer.hpp"

#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <vector>

using namespace swiftimpute;

static void dump(const std::string& path, const void* p, size_t n) {
    std::ofstream o(path, std::ios::binary);
    o.write(static_cast<const char*>(p), n);
}

int main(int argc, char** argv) {
    if (argc == 4 && std::string(argv[1]) == "loadbin") {
        try {
            if (std::string(argv[2]) == "panel") {
                auto p = ReferencePanel::load_binary(argv[3]);
                std::printf("panel M=%u N=%u\n", p->num_markers(), p->num_haplotypes());
            } else {
                auto t = TargetData::load_binary(argv[3]);
                std::printf("target M=%u B=%u\n", t->num_markers(), t->num_samples());
            }
            return 0;
        } catch (const ImputationError& e) {
            std::printf("ImputationError: %s\n", e.what());
            return 11;
        } catch (const std::exception& e) {
            std::printf("error: %s\n", e.what());
            return 12;
        }
    }
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
            tgt->save_binary(pre + ".sitarget");
            auto tback = TargetData::load_binary(pre + ".sitarget");
            const bool tsame = tback->num_markers() == tgt->num_markers() &&
                               tback->num_samples() == tgt->num_samples() &&
                               std::memcmp(tback->genotype_likelihoods(), tgt->genotype_likelihoods(),
                                           (size_t)tgt->num_samples() * tgt->num_markers() *
                                               sizeof(GenotypeLikelihoods)) == 0 &&
                               tback->samples().back().id == tgt->samples().back().id &&
                               tback->markers().back().pos == tgt->markers().back().pos;
            bool refused = false;  // each loader refuses the other's file
            try {
                ReferencePanel::load_binary(pre + ".sitarget");
            } catch (const ImputationError&) {
                refused = true;
            }
            try {
                TargetData::load_binary(pre + ".sipanel");
                refused = false;
            } catch (const ImputationError&) {
            }
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
            std::printf("M=%u N=%u B=%u roundtrip=%d target_roundtrip=%d refused=%d info0=%.4f\n",
                        ref->num_markers(), ref->num_haplotypes(), tgt->num_samples(), same ? 1 : 0, tsame ? 1 : 0,
                        refused ? 1 : 0, r.get_info_score(0));
            return same && tsame && refused ? 0 : 3;
        }
        if (cmd == "multi") {
            std::vector<int> devices;
            for (const char* c = argv[4]; *c;) {
                devices.push_back(std::atoi(c));
                while (*c && *c != ',') ++c;
                if (*c == ',') ++c;
            }
            ImputationConfig cfg;
            cfg.deterministic = std::atoi(argv[6]) != 0;
            cfg.hmm_params.num_states = (uint32_t)std::atoi(argv[7]);
            cfg.hmm_params.ne = (uint32_t)std::atoi(argv[8]);
            MultiGPUImputer multi(*ref, devices, cfg);
            multi.build_indices();
            auto res = multi.impute(*tgt);
            Imputer one(*ref, cfg);
            one.build_index();
            auto want = one.impute(*tgt);
            const size_t n = (size_t)res->num_samples() * res->num_markers();
            bool same = std::memcmp(res->haplotype0(0), want->haplotype0(0), 2 * n) == 0;
            for (sample_t s = 0; s < res->num_samples(); ++s)
                for (marker_t m = 0; m < res->num_markers(); ++m) {
                    prob_t a[3], b[3];
                    res->get_probabilities(s, m, a);
                    want->get_probabilities(s, m, b);
                    same = same && std::memcmp(a, b, sizeof a) == 0 &&
                           res->get_posterior_dosage(s, m) == want->get_posterior_dosage(s, m);
                }
            for (marker_t m = 0; m < res->num_markers(); ++m)
                same = same && res->get_info_score(m) == want->get_info_score(m);
            const std::string pre = argv[5];
            std::vector<float> ds(n);
            for (sample_t s = 0; s < res->num_samples(); ++s)
                for (marker_t m = 0; m < res->num_markers(); ++m)
                    ds[(size_t)s * res->num_markers() + m] = res->get_posterior_dosage(s, m);
            dump(pre + ".dosage", ds.data(), n * 4);
            dump(pre + ".haps", res->haplotype0(0), 2 * n);
            std::printf("multi ok: replicas=%u identical=%d\n", multi.num_gpus(), same ? 1 : 0);
            return same ? 0 : 3;
        }
        if (cmd == "index") {
            // build, store to a file, and impute again through a second Imputer that loads it
            ImputationConfig cfg;
            cfg.hmm_params.num_states = 8;
            Imputer a(*ref, cfg);
            a.build_index();
            a.save_index(argv[4]);
            auto ra = a.impute(*tgt);
            Imputer b(*ref, cfg);
            b.load_index(argv[4]);
            auto rb = b.impute(*tgt);
            const size_t n = (size_t)ra->num_samples() * ra->num_markers();
            const bool same = std::memcmp(ra->haplotype0(0), rb->haplotype0(0), 2 * n) == 0;
            std::printf("index same=%d has_index=%d\n", same ? 1 : 0, b.has_index() ? 1 : 0);
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
