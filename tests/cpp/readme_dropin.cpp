// The reference's README example (README.md:41-47) compiled against the drop-in headers instead
// of the reference's: prints "1 3 2 0". Then a ShockHash2<64> and a ShockHash2Flat<32> over 20000
// keys, each checked to be a minimal perfect hash, a ShockHash<16> over 128-bit hashes, and the
// SIMD format (SIMDShockHash<30>, with and without rotation fitting).
#include <algorithm>
#include <iostream>
#include <string>
#include <vector>
#include "shockhash_b200/ShockHash.h"
#include "shockhash_b200/ShockHash2.h"
#include "shockhash_b200/ShockHash2Flat.h"
#include "shockhash_b200/SIMDShockHash.h"

template <class F> static bool is_mphf(F &f, const std::vector<std::string> &keys) {
    std::vector<char> seen(keys.size(), 0);
    for (const auto &k : keys) {
        size_t v = f(k);
        if (v >= keys.size() || seen[v]) return false;
        seen[v] = 1;
    }
    return true;
}

int main() {
    std::vector<std::string> keys = {"abc", "def", "123", "456"};
    shockhash::ShockHash<30, false> shockHash(keys, 2000);  // ShockHash base case size n=30, bucket size b=2000
    std::cout << shockHash("abc") << " " << shockHash("def") << " " << shockHash("123") << " " << shockHash("456")
              << std::endl;
    std::vector<std::string> many;
    for (int i = 0; i < 20000; i++) many.push_back("key-" + std::to_string(i * 7919));
    shockhash::ShockHash2<64> h2(many, 2000);
    shockhash::ShockHash2Flat<32> hf(many);
    std::cout << (is_mphf(h2, many) ? "ShockHash2 ok" : "ShockHash2 FAIL") << " " << (double)h2.getBits() / many.size()
              << std::endl;
    std::cout << (is_mphf(hf, many) ? "ShockHash2Flat ok" : "ShockHash2Flat FAIL") << std::endl;
    struct hash128 {
        uint64_t first, second;
    };
    std::vector<hash128> hashes;
    uint64_t x = 88172645463325252ull;
    for (int i = 0; i < 5000; i++) {
        x ^= x << 13, x ^= x >> 7, x ^= x << 17;
        uint64_t y = x * 0x9E3779B97F4A7C15ull;
        hashes.push_back({y, x});
    }
    shockhash::ShockHash<16> h1(hashes, 500);
    std::vector<char> seen(hashes.size(), 0);
    bool ok = true;
    for (const auto &h : hashes) {
        size_t v = h1(h);
        ok = ok && v < hashes.size() && !seen[v];
        if (v < hashes.size()) seen[v] = 1;
    }
    std::cout << (ok ? "ShockHash hash128 ok" : "ShockHash hash128 FAIL") << std::endl;
    shockhash::ShockHash<30, true> hr(many, 2000);  // rotation fitting
    std::cout << (is_mphf(hr, many) ? "ShockHash rotation ok" : "ShockHash rotation FAIL") << std::endl;
    shockhash::SIMDShockHash<30, false> hs(many, 2000);
    shockhash::SIMDShockHash<30, true> hsr(many, 2000);
    std::cout << (is_mphf(hs, many) && is_mphf(hsr, many) ? "SIMDShockHash ok" : "SIMDShockHash FAIL") << std::endl;
    return 0;
}
