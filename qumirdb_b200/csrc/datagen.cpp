// datagen.cpp — seeded synthetic inputs with the benchmark configurations'
// shapes and distributions.  Every value is a pure function of (seed,
// stream, row) (SplitMix64 counter generator), so any range of rows can be
// generated in parallel and reproduced exactly.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <thread>
#include <vector>

#include "../../include/qdb_gpu.h"

namespace {

inline uint64_t Mix(uint64_t x) {
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}

inline uint64_t Rand(uint64_t seed, uint64_t stream, uint64_t i) {
    return Mix(Mix(seed * 0x632be59bd9b4e019ull + stream) + i * 0x9e3779b97f4a7c15ull);
}

// Uniform integer in [lo, hi].
inline int64_t Uniform(uint64_t r, int64_t lo, int64_t hi) {
    const unsigned __int128 span = (unsigned __int128)(uint64_t(hi - lo) + 1);
    return lo + int64_t((span * r) >> 64);
}

inline double Unit(uint64_t r) { return double(r >> 11) * (1.0 / 9007199254740992.0); }

template <class F>
void ParallelRows(int64_t rows, F&& f) {
    const int64_t nt = std::max<int64_t>(1, std::min<int64_t>(std::thread::hardware_concurrency(), (rows >> 16) + 1));
    std::vector<std::thread> th;
    for (int64_t t = 0; t < nt; ++t) {
        th.emplace_back([&, t] {
            const int64_t b = rows * t / nt, e = rows * (t + 1) / nt;
            for (int64_t i = b; i < e; ++i) f(i);
        });
    }
    for (auto& x : th) x.join();
}

constexpr int32_t kEpoch = 8035;        // 1992-01-01 in days since 1970-01-01
constexpr int32_t kSpan = 7 * 365;      // seven years of ship dates
constexpr int32_t kStatusCut = 9298;    // later ship dates are still open ('O')

}  // namespace

extern "C" {

void qdb_gen_lineitem(uint64_t seed, int64_t rows, int64_t* qty, int64_t* price, int64_t* disc, int64_t* tax,
                      uint8_t* flag, uint8_t* status, int32_t* shipdate) {
    ParallelRows(rows, [&](int64_t i) {
        qty[i] = Uniform(Rand(seed, 1, i), 1, 50);
        price[i] = Uniform(Rand(seed, 2, i), 90000, 10500000);
        disc[i] = Uniform(Rand(seed, 3, i), 0, 10);
        tax[i] = Uniform(Rand(seed, 4, i), 0, 8);
        const int32_t d = kEpoch + int32_t(Uniform(Rand(seed, 5, i), 0, kSpan - 1));
        shipdate[i] = d;
        const bool open = d > kStatusCut;
        status[i] = open ? 'O' : 'F';
        if (open) {
            flag[i] = 'N';
        } else {
            const int64_t u = Uniform(Rand(seed, 6, i), 0, 99);
            flag[i] = u < 49 ? 'A' : (u < 51 ? 'N' : 'R');
        }
    });
}

void qdb_gen_join(uint64_t seed, int64_t build_rows, int64_t probe_rows, int64_t fk_domain, int64_t* b_key,
                  int64_t* b_payload, int32_t* b_attr, int64_t* p_fk, int64_t* p_value) {
    // Build keys: a seeded Fisher-Yates permutation of 1..build_rows.
    for (int64_t i = 0; i < build_rows; ++i) b_key[i] = i + 1;
    for (int64_t i = build_rows - 1; i > 0; --i) {
        const int64_t j = Uniform(Rand(seed, 10, uint64_t(i)), 0, i);
        std::swap(b_key[i], b_key[j]);
    }
    ParallelRows(build_rows, [&](int64_t i) {
        b_payload[i] = Uniform(Rand(seed, 11, i), 1, 1000000);
        b_attr[i] = int32_t(Uniform(Rand(seed, 12, i), 0, 99));
    });
    ParallelRows(probe_rows, [&](int64_t i) {
        p_fk[i] = Uniform(Rand(seed, 13, i), 1, fk_domain);
        p_value[i] = Uniform(Rand(seed, 14, i), 1, 10000);
    });
}

void qdb_gen_zipf(uint64_t seed, int64_t rows, int64_t distinct, double s, int64_t* key, int64_t* a, double* x) {
    // Inverse CDF over ranks 1..distinct with P(k) proportional to k^-s; the
    // rank goes through a seeded bijection of 64-bit words so keys spread.
    std::vector<double> cdf(size_t(std::max<int64_t>(distinct, 1)));
    double acc = 0.0;
    for (int64_t k = 0; k < distinct; ++k) {
        acc += std::pow(double(k + 1), -s);
        cdf[size_t(k)] = acc;
    }
    const double total = acc;
    const uint64_t salt = Mix(seed ^ 0x5a5a5a5a5a5a5a5aull);
    ParallelRows(rows, [&](int64_t i) {
        const double u = Unit(Rand(seed, 20, i)) * total;
        const int64_t rank = int64_t(std::upper_bound(cdf.begin(), cdf.end(), u) - cdf.begin());
        key[i] = int64_t(Mix(uint64_t(std::min(rank, distinct - 1)) ^ salt));
        a[i] = Uniform(Rand(seed, 21, i), -1000000, 1000000);
        x[i] = Unit(Rand(seed, 22, i));
    });
}

void qdb_gen_sort(uint64_t seed, int64_t rows, int64_t* k1, int32_t* k2, int64_t* rowid) {
    ParallelRows(rows, [&](int64_t i) {
        k1[i] = int64_t(Rand(seed, 30, i));
        k2[i] = int32_t(Uniform(Rand(seed, 31, i), 0, 100000));
        if (rowid) rowid[i] = i;
    });
}

}  // extern "C"
