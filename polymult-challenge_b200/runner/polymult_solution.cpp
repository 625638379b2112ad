// polymult_solution.cpp -- point-directory runner: answers every case of a point directory
// with this library's fherma_init / fherma_run / fherma_free.
//
//     polymult_solution <point directory>
//
// The directory format is the challenge harness's (main.cpp:1-15 of the reference describes
// it): manifest.json holds the point ("N", "W", "L") and the number of "cases";
// point/q.bin holds q as L little-endian u32 limbs; cases/NNNNNN/{a,b}.bin hold the operands
// as N x L limbs.  The runner writes out/NNNNNN/c.bin and out/results.json =
// {"init_s": s, "cases": [{"i": i, "seconds": s, "status": "ok"}, ...]}, rewritten after every
// case so that a run that is killed keeps the cases it finished; a case that throws is
// recorded as {"i": i, "seconds": null, "status": "crashed", "note": "<first 200 chars>"}.
// Only fherma_run is inside the timed window.  Files written by the reference's own harness
// and by this runner are interchangeable (the oracle's point writer produces both inputs).
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "fherma_abi.h"

namespace fs = std::filesystem;

namespace {

std::string load_file(const fs::path& p) {
    std::ifstream in(p, std::ios::binary);
    if (!in) throw std::runtime_error("cannot read " + p.string());
    std::stringstream ss;
    ss << in.rdbuf();
    return ss.str();
}

// the value of "key" in the flat manifest object (numbers only)
long long manifest_int(const std::string& json, const char* key) {
    const std::string k = std::string("\"") + key + "\"";
    const size_t at = json.find(k);
    if (at == std::string::npos) throw std::runtime_error(std::string("manifest.json has no ") + key);
    const size_t colon = json.find(':', at + k.size());
    if (colon == std::string::npos) throw std::runtime_error(std::string("manifest.json: malformed ") + key);
    return std::strtoll(json.c_str() + colon + 1, nullptr, 10);
}

std::vector<uint32_t> load_words(const fs::path& p, size_t words) {
    const std::string raw = load_file(p);
    if (raw.size() != words * 4)
        throw std::runtime_error(p.filename().string() + ": " + std::to_string(raw.size()) + " bytes, expected " +
                                 std::to_string(words * 4));
    std::vector<uint32_t> v(words);
    std::memcpy(v.data(), raw.data(), raw.size());
    return v;
}

std::string case_dir(size_t i) {
    char buf[16];
    std::snprintf(buf, sizeof buf, "%06zu", i);
    return buf;
}

std::string seconds_str(double s) {
    char buf[64];
    std::snprintf(buf, sizeof buf, "%.9f", s);
    return buf;
}

std::string escaped_note(const std::string& why) {
    std::string out;
    for (char c : why.substr(0, 200)) {
        if (c == '"' || c == '\\') out += '\\';
        out += c == '\n' ? ' ' : c;
    }
    return out;
}

void write_results(const fs::path& out, double init_s, const std::vector<std::string>& entries) {
    std::ofstream f(out / "results.json");
    f << "{\"init_s\":" << seconds_str(init_s) << ",\"cases\":[";
    for (size_t i = 0; i < entries.size(); ++i) f << (i ? "," : "") << entries[i];
    f << "]}";
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 2) {
        std::cerr << "usage: polymult_solution <point directory>\n";
        return 2;
    }
    try {
        const fs::path root = argv[1];
        const std::string manifest = load_file(root / "manifest.json");
        fherma::Point p;
        p.N = (uint32_t)manifest_int(manifest, "N");
        p.W = (uint32_t)manifest_int(manifest, "W");
        p.L = (uint32_t)manifest_int(manifest, "L");
        p.q.shape = {(int64_t)p.L};
        p.q.data = load_words(root / "point" / "q.bin", p.L);
        const size_t ncases = (size_t)manifest_int(manifest, "cases");
        const fs::path out = root / "out";
        fs::create_directories(out);

        using clk = std::chrono::steady_clock;
        const auto t0 = clk::now();
        void* st = fherma_init(p);
        const double init_s = std::chrono::duration<double>(clk::now() - t0).count();
        std::vector<std::string> entries;
        write_results(out, init_s, entries);
        const size_t words = (size_t)p.N * p.L;
        for (size_t i = 0; i < ncases; ++i) {
            const fs::path cd = root / "cases" / case_dir(i);
            std::string entry;
            try {
                fherma::Inputs in;
                in.a.shape = in.b.shape = {(int64_t)p.N, (int64_t)p.L};
                in.a.data = load_words(cd / "a.bin", words);
                in.b.data = load_words(cd / "b.bin", words);
                const auto t1 = clk::now();
                fherma::Outputs res = fherma_run(st, in);
                const double s = std::chrono::duration<double>(clk::now() - t1).count();
                const fs::path od = out / case_dir(i);
                fs::create_directories(od);
                std::ofstream f(od / "c.bin", std::ios::binary);
                f.write(reinterpret_cast<const char*>(res.c.data.data()), (std::streamsize)(res.c.data.size() * 4));
                if (!f) throw std::runtime_error("writing out/" + case_dir(i) + "/c.bin failed");
                entry = "{\"i\":" + std::to_string(i) + ",\"seconds\":" + seconds_str(s) + ",\"status\":\"ok\"}";
            } catch (const std::exception& e) {
                entry = "{\"i\":" + std::to_string(i) + ",\"seconds\":null,\"status\":\"crashed\",\"note\":\"" +
                        escaped_note(e.what()) + "\"}";
            }
            entries.push_back(entry);
            write_results(out, init_s, entries);
        }
        fherma_free(st);
        write_results(out, init_s, entries);
    } catch (const std::exception& e) {
        std::cerr << "polymult_solution: " << e.what() << "\n";
        return 1;
    }
    return 0;
}
