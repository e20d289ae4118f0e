// gen.h -- TEST INFRASTRUCTURE ONLY: the benchmark configurations' relation
// generator, restated for the reference harnesses (oracle/ref/harness.cpp for
// hashing/, oracle/ref/harness_sort.cpp for sorting/), so the reference joins
// run on exactly the relations the benchmark gives the GPU library
// (alliancedb_b200/csrc/datagen.cuh; tests/test_oracle.py checks the two
// produce the same arrays).  Tuple is the reference's tuple_t of either tree.
#pragma once

#include <stdint.h>

#include <cmath>
#include <fstream>
#include <thread>
#include <vector>

static uint64_t fmix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
static uint64_t mix3(uint64_t seed, uint64_t stream, uint64_t i) {
    return fmix64(fmix64(seed + stream * 0x632BE59BD9B4E019ULL) ^ (i * 0x9E3779B97F4A7C15ULL + 1));
}
struct Feistel {
    uint64_t n, hmask;
    uint32_t half;
    uint64_t k[4];
    Feistel(uint64_t n_, uint64_t seed) : n(n_) {
        uint32_t bits = 2;
        while (bits < 64 && (1ULL << bits) < n_) bits++;
        bits = (bits + 1) & ~1u;
        half = bits / 2;
        hmask = (1ULL << half) - 1;
        for (int r = 0; r < 4; r++) k[r] = mix3(seed, 1000 + r, 0);
    }
    uint64_t once(uint64_t x) const {
        uint64_t L = x >> half, R = x & hmask;
        for (int r = 0; r < 4; r++) {
            const uint64_t t = R;
            R = L ^ (fmix64(k[r] ^ R) & hmask);
            L = t;
        }
        return (L << half) | R;
    }
    uint64_t operator()(uint64_t i) const {
        uint64_t x = once(i);
        while (x >= n) x = once(x);
        return x;
    }
};

// Zipf(theta) rank in [0, n) by rejection-inversion (Hormann and Derflinger,
// ACM TOMACS 6(3), 1996), as the benchmark generator draws it.
struct ZipfRank {
    double s, n, hx1, hn, sq;
    static double helper1(double x) { return fabs(x) > 1e-8 ? log1p(x) / x : 1.0 - x * (0.5 - x * (1.0 / 3.0 - 0.25 * x)); }
    static double helper2(double x) {
        return fabs(x) > 1e-8 ? expm1(x) / x : 1.0 + x * 0.5 * (1.0 + x * (1.0 / 3.0) * (1.0 + 0.25 * x));
    }
    double h(double x) const { return exp(-s * log(x)); }
    double hint(double x) const {
        const double lx = log(x);
        return helper2((1.0 - s) * lx) * lx;
    }
    double hinv(double x) const {
        double t = x * (1.0 - s);
        if (t < -1.0) t = -1.0;
        return exp(helper1(t) * x);
    }
    ZipfRank(uint64_t n_, double theta) : s(theta), n((double)n_) {
        hx1 = hint(1.5) - 1.0;
        hn = hint(n + 0.5);
        sq = 2.0 - hinv(hint(2.5) - h(2.0));
    }
    uint64_t sample(uint64_t seed, uint64_t j) const {
        for (uint32_t attempt = 0; attempt < 64; attempt++) {
            const double u01 = ((mix3(seed, 7, j * 64 + attempt) >> 11) + 1) * (1.0 / 9007199254740992.0);
            const double u = hn + u01 * (hx1 - hn);
            const double x = hinv(u);
            double kd = floor(x + 0.5);
            if (kd < 1.0) kd = 1.0;
            if (kd > n) kd = n;
            if (kd - x <= sq || u >= hint(kd + 0.5) - h(kd)) return (uint64_t)kd - 1;
        }
        return 0;
    }
};

template <class F>
static void par_for(uint64_t n, F f) {
    unsigned nt = std::thread::hardware_concurrency();
    if (nt == 0 || n < (1u << 16)) nt = 1;
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; t++) {
        const uint64_t b = n * t / nt, e = n * (t + 1) / nt;
        th.emplace_back([=] { for (uint64_t i = b; i < e; i++) f(i); });
    }
    for (auto &x : th) x.join();
}

// R: key = 1 + perm_1(i), payload = i.  S: payload = j, key = R.key[idx_j], idx_j
// uniform over 0..n-1 (theta 0) or rank_perm(Zipf(theta) rank) (seed 2).
template <class Tuple>
static void gen_pkfk(uint64_t n, double theta, std::vector<Tuple> &R, std::vector<Tuple> &S) {
    R.resize(n);
    S.resize(n);
    Feistel perm(n ? n : 1, 1);
    par_for(n, [&](uint64_t i) {
        R[i].payloadID = (int32_t)i;
        R[i].key = (int32_t)(1 + perm(i));
    });
    Feistel rank_perm(n ? n : 1, 2 ^ 0x5A5A5A5A5A5A5A5AULL);
    ZipfRank z(n ? n : 1, theta > 0 ? theta : 1.0);
    par_for(n, [&](uint64_t j) {
        const uint64_t idx = theta > 0 ? rank_perm(z.sample(2, j))
                                       : (uint64_t)(((unsigned __int128)mix3(2, 3, j) * n) >> 64);
        S[j].payloadID = (int32_t)j;
        S[j].key = R[idx].key;
    });
}

template <class Tuple>
static bool read_rel(const char *path, std::vector<Tuple> &out) {
    std::ifstream f(path, std::ios::binary | std::ios::ate);
    if (!f) return false;
    const std::streamsize bytes = f.tellg();
    f.seekg(0);
    out.resize(bytes / sizeof(Tuple));
    f.read(reinterpret_cast<char *>(out.data()), (std::streamsize)(out.size() * sizeof(Tuple)));
    return (bool)f;
}

