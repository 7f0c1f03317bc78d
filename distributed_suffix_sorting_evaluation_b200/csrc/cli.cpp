// dcx_cli: command line front end with the flag surface of lightweight_dcx's
// `cli` (lightweight_dcx/src/executables/cli.cpp:149-305), running the suffix
// array construction on one GPU through the C ABI of libdcxgpu.
//
//   read_input      cli.cpp:393-415 (file, cut to --textsize like mpi/io.hpp:45-47;
//                   --input random generates --textsize chars over 1..--alphabet_size)
//   compute_sa      cli.cpp:655-689 (alphabet remap + DCX with or without packing)
//   check_sa        cli.cpp:700-727 (--check prints "SA_ok=1" when correct)
//   write_sa        cli.cpp:691-698 (--output: raw uint40 little endian, or --sa-width 64)
//   --sa-input F    (GPU addition) with --check: check the SA in file F, in
//                   that raw layout, instead of building one
//   JSON            cli.cpp:804-817 (<path>_timer.json / <path>_counter.json)
// Flags that tune the distributed sorters or the bucket scheme of the reference
// (--atomic-sorter, --buckets-*, --splitter-*, ...) are accepted and recorded in
// the JSON config; they do not change anything on one GPU.
#include <stdint.h>
#include <sys/stat.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <map>
#include <random>
#include <set>
#include <sstream>
#include <string>
#include <vector>

#include "dcx_gpu.h"

namespace {

const std::set<std::string> kValueFlags = {
    "--input", "--textsize", "--iteration", "--alphabet_size", "--output", "--json-output-path", "--seed", "--dcx",
    "--discarding-threshold", "--num-samples-splitters", "--buckets-sample-phase", "--buckets-merging-phase",
    "--buckets-phase3", "--samples-buckets-phase3", "--avg-chunks-pe", "--pack-extra-words", "--atomic-sorter",
    "--ams-levels", "--splitter-sampling", "--splitter-sorting", "--string-sorter", "--memory_seq_string_sorter",
    "--lcp-compression-threshold", "--inital-prefix-length",
    // GPU additions
    "--sa-width", "--device", "--hbm-budget", "--recursion-dc", "--sa-input"};
const std::set<std::string> kBoolFlags = {
    "--check", "--use-random-sampling-splitters", "--balance-blocks-space-efficient-sort", "--use-randomized-chunks",
    "--use-char-packing-samples", "--use-char-packing-merging", "--rearrange-buckets-balanced", "--use-robust-tie-break",
    "--use-compressed-buckets", "--use-string-sort", "--use-string-sort-tie-breaking-phase1",
    "--use-string-sort-tie-breaking-phase4", "--use-loser-tree", "--use-rquick-for-splitters",
    "--use-binary-search-for-splitters", "--use-lcp-compression", "--use-prefix-doubling",
    // GPU additions
    "--dry-run"};
// flags whose value changes what the GPU build computes or writes
const std::set<std::string> kHonoured = {"--input", "--textsize", "--output", "--json-output-path", "--dcx", "--check",
                                         "--seed", "--alphabet_size", "--use-char-packing-samples",
                                         "--use-char-packing-merging", "--discarding-threshold", "--pack-extra-words",
                                         "--iteration", "--sa-width", "--device", "--hbm-budget", "--recursion-dc",
                                         "--dry-run", "--sa-input"};

struct Args {
    std::map<std::string, std::string> v;
    std::vector<std::string> errors;
    bool has(const std::string& k) const { return v.count(k) != 0; }
    std::string get(const std::string& k, const std::string& d = "") const {
        auto it = v.find(k);
        return it == v.end() ? d : it->second;
    }
};

Args parse(int argc, char** argv) {
    Args a;
    for (int i = 1; i < argc; i++) {
        std::string s = argv[i];
        std::string val;
        bool inline_val = false;
        const size_t eq = s.find('=');
        if (s.rfind("--", 0) == 0 && eq != std::string::npos) {
            val = s.substr(eq + 1);
            s = s.substr(0, eq);
            inline_val = true;
        }
        if (kBoolFlags.count(s)) {
            a.v[s] = inline_val ? val : "1";
        } else if (kValueFlags.count(s)) {
            if (!inline_val) {
                if (i + 1 >= argc) {
                    a.errors.push_back(s + " needs a value");
                    break;
                }
                val = argv[++i];
            }
            a.v[s] = val;
        } else {
            a.errors.push_back("unknown option " + s);
        }
    }
    return a;
}

std::string json_escape(const std::string& s) {
    std::string o;
    for (char ch : s) {
        if (ch == '"' || ch == '\\') o += '\\';
        o += ch;
    }
    return o;
}

void write_json(const std::string& path, const std::vector<std::pair<std::string, double>>& entries,
                const std::vector<std::pair<std::string, std::string>>& config, bool nested_timer) {
    std::ofstream out(path);
    out << "[\n{\n  \"data\": {\n    \"root\": {\n      \"statistics\": {\n      },\n";
    if (nested_timer) {
        // total_time -> {compress_alphabet, pdcx -> phases}, plus io / check_SA at top level
        out << "      \"io\": {\"statistics\": {\"max\": [" << entries[0].second << "]}},\n";
        out << "      \"total_time\": {\n        \"statistics\": {\"max\": [" << entries[1].second << "]},\n";
        out << "        \"compress_alphabet\": {\"statistics\": {\"max\": [" << entries[2].second << "]}},\n";
        out << "        \"pdcx\": {\n          \"statistics\": {\"max\": [" << entries[3].second << "]},\n";
        for (size_t i = 4; i < entries.size(); i++) {
            out << "          \"" << entries[i].first << "\": {\"statistics\": {\"max\": [" << entries[i].second
                << "]}}" << (i + 1 < entries.size() ? "," : "") << "\n";
        }
        out << "        }\n      }\n";
    } else {
        for (size_t i = 0; i < entries.size(); i++) {
            out << "      \"" << entries[i].first << "\": {\"statistics\": {\"max\": [" << (int64_t)entries[i].second
                << "]}}" << (i + 1 < entries.size() ? "," : "") << "\n";
        }
    }
    out << "    }\n  },\n  \"config\": {\n";
    for (size_t i = 0; i < config.size(); i++)
        out << "    \"" << json_escape(config[i].first) << "\":\"" << json_escape(config[i].second) << "\""
            << (i + 1 < config.size() ? "," : "") << "\n";
    out << "  }\n}\n]\n";
}

int fail(const std::string& msg) {
    std::cerr << msg << std::endl;
    return 1;
}

}  // namespace

int main(int argc, char** argv) {
    Args a = parse(argc, argv);
    if (!a.errors.empty()) {
        for (auto& e : a.errors) std::cerr << e << "\n";
        return 1;
    }
    const std::string input = a.get("--input");
    const uint64_t textsize = std::stoull(a.get("--textsize", "0"));
    std::string dcx = a.get("--dcx", "dc39");
    const int X = std::atoi(dcx.c_str() + (dcx.rfind("dc", 0) == 0 ? 2 : 0));
    const bool packing = a.has("--use-char-packing-samples") || a.has("--use-char-packing-merging");
    const int width = std::atoi(a.get("--sa-width", "40").c_str());
    const int device = std::atoi(a.get("--device", "0").c_str());
    const double discarding = std::stod(a.get("--discarding-threshold", "0.7"));
    if (a.get("--pack-extra-words", "0") != "0") return fail("--pack-extra-words: only 0 is supported (cli.cpp:675-682)");
    if (!(width == 32 || width == 40 || width == 64)) return fail("--sa-width must be 32, 40 or 64");
    if (dcx_dc_table(X, nullptr, nullptr, nullptr, nullptr) != DCX_OK) return fail("unsupported --dcx " + dcx);
    if (a.has("--sa-input") && !a.has("--check")) return fail("--sa-input needs --check");

    std::vector<std::pair<std::string, std::string>> config;
    for (auto& kv : a.v) config.emplace_back(kv.first.substr(2), kv.second);
    config.emplace_back("algorithm", "DCX");
    config.emplace_back("dcx_variant", "dc" + std::to_string(X));
    config.emplace_back("num_pe", "1");
    config.emplace_back("backend", "B200 GPU");
    std::vector<std::string> ignored;
    for (auto& kv : a.v)
        if (!kHonoured.count(kv.first)) ignored.push_back(kv.first);

    if (a.has("--dry-run")) {
        std::cout << "{\"dcx\": " << X << ", \"packing\": " << (packing ? "true" : "false") << ", \"sa_width\": "
                  << width << ", \"textsize\": " << textsize << ", \"input\": \"" << json_escape(input)
                  << "\", \"ignored\": [";
        for (size_t i = 0; i < ignored.size(); i++) std::cout << (i ? ", " : "") << "\"" << ignored[i] << "\"";
        std::cout << "]}" << std::endl;
        return 0;
    }
    for (auto& f : ignored) std::cout << "note: " << f << " has no effect on a single GPU" << std::endl;

    // ---- read_input (cli.cpp:393-415)
    auto t_io0 = std::chrono::steady_clock::now();
    std::vector<uint8_t> text;
    if (input == "random") {
        const uint64_t sigma = std::stoull(a.get("--alphabet_size", "2"));
        std::mt19937 rng((uint32_t)std::stoull(a.get("--seed", "0")));  // util/random.hpp:7-15
        std::uniform_int_distribution<uint32_t> dist(1, (uint32_t)sigma);
        text.resize(textsize);
        for (auto& c : text) c = (uint8_t)dist(rng);
    } else {
        struct stat stt;
        if (input.empty() || stat(input.c_str(), &stt) != 0)
            return fail("File " + input + " does not exist!");
        uint64_t size = (uint64_t)stt.st_size;
        if (textsize > 0) size = std::min<uint64_t>(size, textsize);
        text.resize(size);
        std::ifstream in(input, std::ios::binary);
        in.read(reinterpret_cast<char*>(text.data()), (std::streamsize)size);
        if ((uint64_t)in.gcount() != size) return fail("short read of " + input);
    }
    const double io_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_io0).count();
    const uint64_t n = text.size();

    // ---- compute_sa (cli.cpp:655-689)
    dcx_ctx* ctx = nullptr;
    int rc = dcx_ctx_create(&ctx, device, std::stoull(a.get("--hbm-budget", "0")));
    if (rc != DCX_OK) return fail(std::string("dcx_ctx_create: ") + dcx_strerror(rc));
    // ---- --sa-input: check an existing SA file (e.g. the reference cli's --output) instead of building
    const std::string sa_input = a.get("--sa-input");
    if (!sa_input.empty()) {
        int ok = 0;
        auto c0 = std::chrono::steady_clock::now();
        rc = dcx_check_sa_file(ctx, text.data(), n, sa_input.c_str(), width, DCX_HOST_PTRS, &ok);
        const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - c0).count();
        dcx_ctx_destroy(ctx);
        if (rc != DCX_OK) return fail(std::string("dcx_check_sa_file: ") + dcx_strerror(rc));
        std::cout << (ok ? "Correct SA!" : "ERROR: Not a correct SA!") << "\n";
        std::cout << "SA_ok=" << ok << "\n";
        std::cout << "check_time=" << s << "\n";
        return 0;
    }
    dcx_set_option(ctx, "discarding_threshold", discarding);
    if (a.has("--recursion-dc")) dcx_set_option(ctx, "recursion_dc", std::stod(a.get("--recursion-dc")));
    std::vector<uint8_t> sa(n * (width / 8) + 1);
    auto t0 = std::chrono::steady_clock::now();
    rc = dcx_build_sa(ctx, text.data(), n, X, width, sa.data(), DCX_HOST_PTRS | (packing ? 0u : DCX_NO_PACKING));
    const double total_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (rc != DCX_OK) {
        dcx_ctx_destroy(ctx);
        return fail(std::string("dcx_build_sa: ") + dcx_strerror(rc));
    }
    dcx_stats st{};
    dcx_get_stats(ctx, &st);
    std::cout << "input_alphabet_size=" << st.sigma << "\n";
    std::cout << "total_time=" << total_s << " device_ms=" << st.ms_total << " GiB/s="
              << (total_s > 0 ? n / total_s / (1024.0 * 1024 * 1024) : 0) << "\n";
    std::cout << "levels=" << st.levels << " level0_samples=" << st.level0_samples
              << " level0_highest_rank=" << st.level0_last_rank << " level0_recursion=" << st.level0_recursion << "\n";

    // ---- check_sa (cli.cpp:700-727)
    double check_s = 0;
    if (a.has("--check")) {
        auto c0 = std::chrono::steady_clock::now();
        int ok = 0;
        rc = dcx_check_sa(ctx, text.data(), n, sa.data(), width, DCX_HOST_PTRS, &ok);
        check_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - c0).count();
        if (rc != DCX_OK) {
            dcx_ctx_destroy(ctx);
            return fail(std::string("dcx_check_sa: ") + dcx_strerror(rc));
        }
        std::cout << (ok ? "Correct SA!" : "ERROR: Not a correct SA!") << "\n";
        std::cout << "SA_ok=" << ok << "\n";
    }

    // ---- write_sa (cli.cpp:691-698, mpi/io.hpp:80-98)
    const std::string output = a.get("--output");
    if (!output.empty()) {
        std::cout << "Writing the SA to " << output << "\n";
        std::ofstream out(output, std::ios::binary);
        out.write(reinterpret_cast<const char*>(sa.data()), (std::streamsize)(n * (width / 8)));
        if (!out) {
            dcx_ctx_destroy(ctx);
            return fail("cannot write " + output);
        }
        std::cout << "Finished writing the SA \n";
    }

    // ---- JSON logs (cli.cpp:804-817), phase names of pdcx.hpp:544,659,741,778
    const std::string jp = a.get("--json-output-path");
    if (!jp.empty()) {
        std::vector<std::pair<std::string, double>> timers = {
            {"io", io_s},
            {"total_time", total_s},
            {"compress_alphabet", st.ms_phase0 / 1000.0},
            {"pdcx", (st.ms_phase12 + st.ms_phase3 + st.ms_phase4) / 1000.0},
            {"phase_01_02_samples_ranks", st.ms_phase12 / 1000.0},
            {"phase_03_recursion", st.ms_phase3 / 1000.0},
            {"phase_04_merge", st.ms_phase4 / 1000.0},
        };
        if (a.has("--check")) timers.emplace_back("check_SA", check_s);
        write_json(jp + "_timer.json", timers, config, true);
        std::vector<std::pair<std::string, double>> counters = {
            {"text_size", (double)n},
            {"input_alphabet_size", (double)st.sigma},
            {"recursion_levels", (double)st.levels},
            {"level0_samples", (double)st.level0_samples},
            {"level0_highest_rank", (double)st.level0_last_rank},
            {"device_peak_bytes", (double)st.peak_bytes},
            {"kernel_launches", (double)st.kernel_launches},
            {"radix_passes", (double)st.radix_passes},
        };
        write_json(jp + "_counter.json", counters, config, false);
    }
    dcx_ctx_destroy(ctx);
    return 0;
}
