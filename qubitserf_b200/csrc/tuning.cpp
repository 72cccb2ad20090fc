#include "tuning.hpp"

#include <dlfcn.h>

#include <algorithm>
#include <cctype>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <string>

namespace qsfb {

namespace {

bool set_key(Tuning& t, const std::string& key, const std::string& val) {
    char* end = nullptr;
    const double v = std::strtod(val.c_str(), &end);
    if (end == val.c_str()) return false;
    const long long iv = (long long)v;
    if (key == "tc_shape") t.tc_shape = iv == 0 ? 0 : 1;
    else if (key == "tc_job_tiles.small") t.tc_job_tiles_small = (int)std::max(1ll, std::min(64ll, iv));
    else if (key == "tc_job_tiles.large") t.tc_job_tiles_large = (int)std::max(1ll, std::min(64ll, iv));
    else if (key == "tc_small_tiles") t.tc_small_tiles = std::max(0ll, iv);
    else if (key == "cc_jobs_per_warp") t.cc_jobs_per_warp = (int)std::max(1ll, std::min(256ll, iv));
    else if (key == "tc_cost_ratio") t.tc_cost_ratio = std::max(0.0, std::min(4.0, v));
    else if (key == "tc_edge_div") t.tc_edge_div = (int)std::max(1ll, std::min(64ll, iv));
    else if (key == "exec_groups") t.exec_groups = (int)std::max(1ll, std::min(16ll, iv));
    else if (key == "batch_chunks") t.batch_chunks = (int)std::max(1ll, std::min(64ll, iv));
    else if (key == "overlap_groups") t.overlap_groups = (int)std::max(1ll, std::min(16ll, iv));
    else if (key == "batch_first_permille")
        t.batch_first_permille = (int)std::max(0ll, std::min(1000ll, iv));
    else return false;
    return true;
}

// directory of the loaded library (the table ships beside it)
std::string library_dir() {
    Dl_info info;
    if (dladdr((const void*)&tuning, &info) == 0 || !info.dli_fname) return ".";
    const std::string f = info.dli_fname;
    const size_t slash = f.rfind('/');
    return slash == std::string::npos ? "." : f.substr(0, slash);
}

Tuning load() {
    Tuning t;
    const char* env = std::getenv("QSFB_TUNING");
    const std::string path = env ? std::string(env) : library_dir() + "/tuning.txt";
    std::ifstream in(path);
    if (in) {
        std::string line;
        int used = 0;
        while (std::getline(in, line)) {
            const size_t hash = line.find('#');
            if (hash != std::string::npos) line.resize(hash);
            std::istringstream ls(line);
            std::string key, val;
            if (ls >> key >> val) used += set_key(t, key, val) ? 1 : 0;
        }
        if (used) t.source = path;
    }
    static const char* const keys[] = {"tc_shape", "tc_job_tiles.small", "tc_job_tiles.large",
                                       "tc_small_tiles", "cc_jobs_per_warp", "tc_cost_ratio",
                                       "tc_edge_div",
                                       "exec_groups", "batch_chunks", "overlap_groups",
                                       "batch_first_permille"};
    for (const char* k : keys) {
        std::string name = "QSFB_TUNE_";
        for (const char* c = k; *c; ++c) name += *c == '.' ? '_' : (char)std::toupper(*c);
        if (const char* v = std::getenv(name.c_str()))
            if (set_key(t, k, v)) t.source += " + " + name;
    }
    return t;
}

}  // namespace

const Tuning& tuning() {
    static const Tuning t = load();
    return t;
}

int tc_job_tiles_for(unsigned long long tiles) {
    const Tuning& t = tuning();
    return tiles < (unsigned long long)t.tc_small_tiles ? t.tc_job_tiles_small : t.tc_job_tiles_large;
}

}  // namespace qsfb
