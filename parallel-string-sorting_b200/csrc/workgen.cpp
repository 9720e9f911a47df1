// workgen.cpp -- seeded synthetic workloads, the algorithmic-byte model and
// output checks of the benchmark (libpsswork.so, host only, OpenMP).
//
// Every generator is counter-based (splitmix64 of seed, stream, index), so
// the output does not depend on the thread count. Arenas are NUL-terminated
// strings packed back to back; offs[i] is the start of string i.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

inline uint64_t mix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

inline uint64_t rnd(uint64_t seed, uint64_t stream, uint64_t i)
{
    return mix64(mix64(seed * 0xD1B54A32D192ED03ull + stream) ^ i);
}

inline double unit(uint64_t r) { return (double)(r >> 11) * (1.0 / 9007199254740992.0); }

constexpr int PREFIXES = 4096;
constexpr int PREFIX_LEN = 48;

}  // namespace

extern "C" {

// ---- random strings over an alphabet, lengths uniform in [lmin, lmax] ------
uint64_t pssw_random_offsets(uint64_t seed, uint64_t n, uint32_t lmin, uint32_t lmax,
                             uint64_t* offs)
{
    uint64_t total = 0;
    const uint64_t span = (uint64_t)lmax - lmin + 1;
    for (uint64_t i = 0; i < n; ++i) {
        offs[i] = total;
        total += lmin + rnd(seed, 0, i) % span + 1;
    }
    return total;
}

void pssw_random_fill(uint64_t seed, uint64_t n, const uint64_t* offs, uint64_t nchars,
                      const uint8_t* alphabet, uint32_t asize, uint8_t* chars)
{
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        const uint64_t end = (i + 1 < (int64_t)n) ? offs[i + 1] : nchars;
        const uint64_t len = end - offs[i] - 1;
        uint8_t* p = chars + offs[i];
        for (uint64_t j = 0; j < len; ++j) p[j] = alphabet[rnd(seed, 1, offs[i] + j) % asize];
        p[len] = 0;
    }
}

// ---- digits: lengths U[1,40] over '0'..'9', packed until the next string
// would exceed `budget` bytes (string + terminator). Returns the count. -----
uint64_t pssw_digits_count(uint64_t seed, uint64_t budget, uint64_t* nchars_out)
{
    uint64_t total = 0, n = 0;
    while (true) {
        const uint64_t len = 1 + rnd(seed, 10, n) % 40;
        if (total + len + 1 > budget) break;
        total += len + 1;
        ++n;
    }
    if (nchars_out) *nchars_out = total;
    return n;
}

void pssw_digits_fill(uint64_t seed, uint64_t n, uint64_t* offs, uint8_t* chars)
{
    uint64_t total = 0;
    for (uint64_t i = 0; i < n; ++i) {
        offs[i] = total;
        total += 1 + rnd(seed, 10, i) % 40 + 1;
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        const uint64_t len = 1 + rnd(seed, 10, i) % 40;
        uint8_t* p = chars + offs[i];
        for (uint64_t j = 0; j < len; ++j) p[j] = (uint8_t)('0' + rnd(seed, 11, offs[i] + j) % 10);
        p[len] = 0;
    }
}

// ---- high-LCP prefixes: one of 4096 random 48-char prefixes ('a'..'z'),
// picked Zipf(s) by rank, then a suffix of length U[8,24] over 'a'..'z'. ----
uint64_t pssw_prefix_offsets(uint64_t seed, uint64_t n, uint64_t* offs)
{
    uint64_t total = 0;
    for (uint64_t i = 0; i < n; ++i) {
        offs[i] = total;
        total += PREFIX_LEN + 8 + rnd(seed, 20, i) % 17 + 1;
    }
    return total;
}

void pssw_prefix_fill(uint64_t seed, uint64_t n, const uint64_t* offs, double zipf_s,
                      uint8_t* chars, uint16_t* prefix_ids)
{
    std::vector<uint8_t> pre((size_t)PREFIXES * PREFIX_LEN);
    for (size_t j = 0; j < pre.size(); ++j) pre[j] = (uint8_t)('a' + rnd(seed, 21, j) % 26);
    std::vector<double> cdf(PREFIXES);
    double acc = 0;
    for (int k = 0; k < PREFIXES; ++k) {
        acc += std::pow((double)(k + 1), -zipf_s);
        cdf[k] = acc;
    }
    for (int k = 0; k < PREFIXES; ++k) cdf[k] /= acc;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        const double u = unit(rnd(seed, 22, i));
        int k = (int)(std::lower_bound(cdf.begin(), cdf.end(), u) - cdf.begin());
        if (k >= PREFIXES) k = PREFIXES - 1;
        if (prefix_ids) prefix_ids[i] = (uint16_t)k;
        const uint64_t slen = 8 + rnd(seed, 20, i) % 17;
        uint8_t* p = chars + offs[i];
        memcpy(p, pre.data() + (size_t)k * PREFIX_LEN, PREFIX_LEN);
        for (uint64_t j = 0; j < slen; ++j) p[PREFIX_LEN + j] = (uint8_t)('a' + rnd(seed, 23, (uint64_t)i * 32 + j) % 26);
        p[PREFIX_LEN + slen] = 0;
    }
}

// ---- DNA-like text: len chars uniform over ACGT, then blocks of length
// U[1 KiB, 10 KiB] copied from a uniformly chosen earlier source into a
// uniformly chosen later target until copy_frac * len bytes were written.
// text must hold len + 1 bytes; text[len] = 0 (the reference's --suffix
// loader turns the trailing byte into NUL). Returns the number of copies. --
uint64_t pssw_dna_text(uint64_t seed, uint64_t len, double copy_frac, uint8_t* text)
{
    static const char acgt[4] = {'A', 'C', 'G', 'T'};
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)len; ++i) text[i] = (uint8_t)acgt[rnd(seed, 30, i) & 3];
    text[len] = 0;
    const uint64_t goal = (uint64_t)(copy_frac * (double)len);
    uint64_t written = 0, copies = 0, draw = 0;
    if (len < 4 * 10240) return 0;
    while (written < goal) {
        const uint64_t L = 1024 + rnd(seed, 31, draw++) % (9 * 1024 + 1);
        const uint64_t dst = L + rnd(seed, 31, draw++) % (len - 2 * L);
        const uint64_t src = rnd(seed, 31, draw++) % (dst - L + 1);
        memmove(text + dst, text + src, L);
        written += L;
        ++copies;
    }
    return copies;
}

// ---- strings of lognormal length: len = round(exp(mu + sigma * z)) clipped
// to [lmin, lmax], z standard normal (Box-Muller on two counter-based
// uniforms). Returns nchars (terminators included). ------------------------
uint64_t pssw_lognormal_offsets(uint64_t seed, uint64_t n, double mu, double sigma,
                                uint32_t lmin, uint32_t lmax, uint64_t* offs)
{
    uint64_t total = 0;
    for (uint64_t i = 0; i < n; ++i) {
        const double u1 = unit(rnd(seed, 40, i)) + 1e-300;
        const double u2 = unit(rnd(seed, 41, i));
        const double z = std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
        double len = std::floor(std::exp(mu + sigma * z) + 0.5);
        if (len < lmin) len = lmin;
        if (len > lmax) len = lmax;
        offs[i] = total;
        total += (uint64_t)len + 1;
    }
    return total;
}

// ---- algorithmic bytes of the sample-sort method for a sorted LCP array --
// Groups at depth 8r are maximal runs of sorted strings whose interior LCPs
// are >= 8r. Every string in a group larger than T at round r costs 52 bytes
// (gather 4+8+8, classify 8, scatter 12+12); every string costs 12 bytes when
// it enters the base case plus the distinguishing chars it still needs there;
// the output costs 8 bytes per string. lcp[0] is ignored.
void pssw_alg_bytes(const uint32_t* lcp, uint64_t n, uint32_t T, uint64_t* out_total,
                    uint64_t* out_rounds_bytes, uint64_t* out_base_bytes, uint32_t* out_max_round)
{
    uint64_t rounds_bytes = 0, base_bytes = 0;
    uint32_t max_round = 0;
    struct Range { uint64_t a, b; uint32_t r; };
    std::vector<Range> stack;
    if (n) stack.push_back({0, n, 0});
    auto need = [&](uint64_t i) -> uint64_t {
        uint64_t l = 0;
        if (i > 0) l = lcp[i];
        if (i + 1 < n) l = std::max<uint64_t>(l, lcp[i + 1]);
        return l + 1;
    };
    while (!stack.empty()) {
        const Range g = stack.back();
        stack.pop_back();
        const uint64_t size = g.b - g.a;
        if (size <= T) {
            const uint64_t d = 8ull * g.r;
            for (uint64_t i = g.a; i < g.b; ++i) {
                const uint64_t nd = need(i);
                base_bytes += 12 + (nd > d ? nd - d : 0);
            }
            continue;
        }
        rounds_bytes += 52ull * size;
        max_round = std::max(max_round, g.r);
        const uint64_t next_depth = 8ull * (g.r + 1);
        uint64_t start = g.a;
        for (uint64_t i = g.a + 1; i <= g.b; ++i) {
            if (i == g.b || lcp[i] < next_depth) {
                stack.push_back({start, i, g.r + 1});
                start = i;
            }
        }
    }
    if (out_total) *out_total = rounds_bytes + base_bytes + 8ull * n;
    if (out_rounds_bytes) *out_rounds_bytes = rounds_bytes;
    if (out_base_bytes) *out_base_bytes = base_bytes;
    if (out_max_round) *out_max_round = max_round;
}

// ---- output checks of a sort (measurement side: the benchmark verifies the
// permutation of a timed sort with these) ----
// The first position p >= 1 where string perm[p-1] > string perm[p]
// (unsigned bytewise, as strcmp), or where an id is out of range; -1 when
// the order holds. chars[nchars - 1] must be NUL.
int64_t pssw_check_sorted(const uint8_t* chars, uint64_t nchars, const uint64_t* offs,
                          const uint32_t* perm, uint64_t n)
{
    int64_t first = INT64_MAX;
    if (nchars == 0 || chars[nchars - 1] != 0) return 0;
#pragma omp parallel for schedule(static) reduction(min : first)
    for (int64_t p = 0; p < (int64_t)n; ++p) {
        const uint32_t b = perm[p];
        if (b >= n || offs[b] >= nchars) {
            first = std::min(first, p);
            continue;
        }
        if (p == 0) continue;
        const uint32_t a = perm[p - 1];
        if (a >= n || offs[a] >= nchars) continue;  // reported at p - 1
        if (strcmp((const char*)chars + offs[a], (const char*)chars + offs[b]) > 0)
            first = std::min(first, p);
    }
    return first == INT64_MAX ? -1 : first;
}

// 1 when perm[0, n) holds every id 0..n-1 exactly once.
int pssw_check_permutation(const uint32_t* perm, uint64_t n)
{
    std::vector<uint8_t> seen(n, 0);
    int ok = 1;
#pragma omp parallel for schedule(static) reduction(min : ok)
    for (int64_t p = 0; p < (int64_t)n; ++p) {
        const uint32_t v = perm[p];
        if (v >= n) {
            ok = 0;
            continue;
        }
        // a byte store races only with another occurrence of v, which the
        // count below reports either way
        seen[v] = 1;
    }
    if (!ok) return 0;
    uint64_t cnt = 0;
#pragma omp parallel for schedule(static) reduction(+ : cnt)
    for (int64_t i = 0; i < (int64_t)n; ++i) cnt += seen[i];
    return cnt == n ? 1 : 0;
}

}  // extern "C"
