// A program written against the reference's API (example.cpp:8-60, benchmark.cpp:31-92),
// compiled against the B200 engine's drop-in header.  It builds MPHFs over u64 keys
// and decimal-string keys on the GPU, checks every function is a bijection onto
// [0, n) by querying every key, and writes the serialised C1 function to a file.
#include <cstdio>
#include <fstream>
#include <string>
#include <type_traits>
#include <vector>

#include "phobic_gpu_mphf.hpp"

using namespace phobicgpu;

struct FileSaver {
    std::ofstream out;
    template <typename T>
    void visit(std::vector<T> &v) {
        size_t n = v.size();
        out.write(reinterpret_cast<const char *>(&n), sizeof(n));
        if constexpr (std::is_trivially_copyable_v<T>) out.write(reinterpret_cast<const char *>(v.data()), n * sizeof(T));
        else for (auto &e : v) visit(e);
    }
    template <typename T>
    void visit(T &v) {
        if constexpr (std::is_trivially_copyable_v<T>) out.write(reinterpret_cast<const char *>(&v), sizeof(T));
        else v.visit(*this);
    }
};

template <typename Mphf, typename K>
static bool bijective(const Mphf &f, const std::vector<K> &keys) {
    std::vector<bool> taken(keys.size(), false);
    for (auto &k : keys) {
        uint32_t h = f(k);
        if (h >= keys.size() || taken[h]) return false;
        taken[h] = true;
    }
    return true;
}

static uint64_t splitmix64(uint64_t seed, uint64_t i) {
    uint64_t z = seed + (i + 1) * 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

int main(int argc, char **argv) {
    const char *dump = argc > 1 ? argv[1] : "c1_interleaved_compact.bin";
    // C1: 1M u64 keys, lambda 5, partition 2048, interleaved compact.
    std::vector<uint64_t> keys(1000000);
    for (size_t i = 0; i < keys.size(); i++) keys[i] = splitmix64(1, i);
    MPHFbuilder builder(MPHFconfig(5.0, 2048));
    FastQueryMphf f;
    HostTimer t = builder.build(keys, f);
    if (!bijective(f, keys)) { std::printf("FAIL u64\n"); return 1; }
    FileSaver s{std::ofstream(dump, std::ios::binary)};
    f.getPilotEncoder().visit(s);
    f.getPartitionOffsetEncoder().visit(s);
    s.out.close();
    std::printf("RESULT keys=u64 n=%zu %s %s\n", keys.size(), f.getResultLine().c_str(), t.getResultStyle(keys.size()).c_str());

    // example.cpp's key set: decimal strings, lambda 4.5, partition 2500, interleaved rice.
    std::vector<std::string> strs;
    for (int i = 0; i < 200000; i++) strs.push_back(std::to_string(i));
    MPHFbuilder sb(MPHFconfig(4.5, 2500));
    MPHF<interleaved_encoder<rice>, diff_partition_encoder<compact>, xxhash> g;
    sb.build(strs, g);
    if (!bijective(g, strs)) { std::printf("FAIL strings\n"); return 1; }
    std::printf("RESULT keys=string n=%zu %s\n", strs.size(), g.getResultLine().c_str());

    // pair keys and pre-hashed Keys, dictionary and dual encoders.
    std::vector<std::pair<uint64_t, uint64_t>> pairs;
    for (uint64_t i = 0; i < 50000; i++) pairs.push_back({splitmix64(7, 2 * i), splitmix64(7, 2 * i + 1)});
    MPHFbuilder pb(MPHFconfig(6.0, 2048));
    MPHF<interleaved_encoder<dictionary>, direct_partition_encoder<compact>, xxhash> h;
    pb.build(pairs, h);
    if (!bijective(h, pairs)) { std::printf("FAIL pairs\n"); return 1; }
    std::vector<Key> pre;
    for (uint64_t i = 0; i < 50000; i++) {
        uint64_t a = splitmix64(8, 2 * i), b = splitmix64(8, 2 * i + 1);
        pre.emplace_back(uint32_t(a), uint32_t(a >> 32), uint32_t(b), uint32_t(b >> 32));
    }
    MPHF<interleaved_encoder_dual<rice, compact>, diff_partition_encoder<compact>, nohash> q;
    pb.build(pre, q);
    if (!bijective(q, pre)) { std::printf("FAIL prehashed\n"); return 1; }
    std::printf("OK\n");
    return 0;
}
