#include "filter_plan.hpp"

#include <algorithm>
#include <cmath>
#include <mutex>

namespace qsfb {

namespace {

constexpr int kFilters[5] = {1, 2, 3, 4, 6};
constexpr int kBits = 128;    // four 32-bit probe words at most
constexpr int kMaxT = 128;

int filter_index(int filt) {
    for (int i = 0; i < 5; ++i)
        if (kFilters[i] == filt) return i;
    return -1;
}

int words_of_filter(int filt) { return filt == 6 ? 4 : filt; }

// cdf[f][nred][t] = P(value of filter f <= t) for a pair over nred random non-pivot bits,
// filled on first use of each (f, nred).
double g_cdf[5][kBits + 1][kMaxT + 1];
std::once_flag g_once[5][kBits + 1];

void fill_table(int fi, int nred) {
    const int filt = kFilters[fi], k = words_of_filter(filt);
    double dist[3 * 32 + 1] = {1.0};
    int top = 0;
    for (int p = 0; p < 32; ++p) {
        int c = 0;   // probe words with a live bit in column p
        for (int j = 0; j < k; ++j) c += (32 * j + p < nred);
        // per-column value distribution
        double pv[4] = {1.0, 0.0, 0.0, 0.0};
        if (filt != 6) {
            if (c > 0) { pv[0] = 1.0 / (double)(1u << c); pv[1] = 1.0 - pv[0]; }
        } else {
            // c live words, count ~ Binomial(c, 1/2); a count of 4 reads as 2
            double bin[5] = {0, 0, 0, 0, 0};
            const double norm = 1.0 / (double)(1u << c);
            double choose = 1.0;
            for (int i = 0; i <= c; ++i) {
                bin[i] = choose * norm;
                choose = choose * (c - i) / (i + 1);
            }
            pv[0] = bin[0]; pv[1] = bin[1]; pv[2] = bin[2] + bin[4]; pv[3] = bin[3];
        }
        double next[3 * 32 + 1] = {0.0};
        for (int s = 0; s <= top; ++s)
            for (int v = 0; v < 4; ++v)
                if (pv[v] != 0.0) next[s + v] += dist[s] * pv[v];
        top = std::min(top + 3, 3 * 32);
        for (int s = 0; s <= top; ++s) dist[s] = next[s];
    }
    double acc = 0.0;
    for (int t = 0; t <= kMaxT; ++t) {
        if (t <= 3 * 32) acc += dist[t];
        g_cdf[fi][nred][t] = std::min(acc, 1.0);
    }
}

}  // namespace

double filter_pass_rate(int filt, int nred, int t) {
    const int fi = filter_index(filt);
    if (fi < 0) return 1.0;
    if (t < 0) return 0.0;
    const int nb = std::min(std::max(nred, 0), kBits);
    std::call_once(g_once[fi][nb], fill_table, fi, nb);
    return g_cdf[fi][nb][std::min(t, kMaxT)];
}

namespace {
// cdf of Binomial(bits, 1/2) for bits <= 128, filled once (static storage, no heap)
double g_ham[kBits + 1][kBits + 1];
std::once_flag g_ham_once;
void fill_ham() {
    for (int bits = 0; bits <= kBits; ++bits) {
        const double lp = -bits * std::log(2.0);
        double acc = 0.0, lc = 0.0;
        for (int t = 0; t <= kBits; ++t) {
            if (t <= bits) {
                if (t > 0) lc += std::log((double)(bits - t + 1) / t);
                acc += std::exp(lc + lp);
            }
            g_ham[bits][t] = std::min(acc, 1.0);
        }
    }
}
}  // namespace

double hamming_pass_rate(int bits, int t) {
    if (t < 0) return 0.0;
    if (t >= bits) return 1.0;
    if (bits > kBits) bits = kBits;   // callers ask for at most four probe words
    std::call_once(g_ham_once, fill_ham);
    return g_ham[bits][t];
}

FilterChoice choose_filter(int HP, int nred, int t, bool zero_test) {
    if (HP <= 1) return {1, zero_test ? 0 : 1};
    if (zero_test) return {2, 0};
    if (HP == 2) return {2, 1};
    // Cost per pair relative to one POPC: the XU pipe (POPC) runs at half the ALU pipe's
    // rate, so a pair costs max(POPCs, ALU ops / 2); ALU ops per pair are the XORs/ORs
    // plus half a three-input minimum (2.5, 3.5, 4.5 and ~9.5).  OR3 is priced a little
    // above OR2 for the contention of two near-saturated pipes.  Added: the exact rescans
    // of a 32-entry chunk that a passing pair causes (~32 * HP POPCs each, 32 chances).
    struct Cand { int filt, popcs; double unit; };
    const Cand cands[4] = {{2, 1, 1.0}, {3, 1, 1.03}, {4, 1, 1.15}, {6, 2, 2.4}};
    const double rescan = 32.0 * 32.0 * HP;
    FilterChoice best{2, 1};
    double best_cost = 1e300;
    for (const Cand& c : cands) {
        const double cost = c.unit + rescan * filter_pass_rate(c.filt, nred, t);
        if (cost < best_cost) { best_cost = cost; best = {c.filt, c.popcs}; }
    }
    return best;
}

}  // namespace qsfb
