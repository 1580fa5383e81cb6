// The serialized pilot layout as a file: the two arrays a build returns, before
// any encoding (the reference hands them straight to Mphf::setData,
// include/phobicGpu/mphf_builder.h:254-289).  Keeping them lets a function be
// re-encoded later with another encoder without building it again.
//
// Little-endian layout:
//   8 bytes   magic "PHBLAYT1"
//   u64       n (keys)
//   u32       partitions
//   u32       buckets per partition
//   u32       partition size P
//   u32       0
//   u32[buckets * partitions]   pilots, bucket-major: pilots[b * partitions + p]
//   u32[partitions + 1]         partition offsets, [0] = 0, last = n
// The Python binding (phobic.save_layout / load_layout) reads and writes the same bytes.
#pragma once

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace phobicgpu {

struct PilotLayout {
    uint64_t n = 0;
    uint32_t partitions = 0;
    uint32_t buckets = 0;
    uint32_t partition_size = 0;
    std::vector<uint32_t> pilots;   // [buckets * partitions]
    std::vector<uint32_t> offsets;  // [partitions + 1]
};

inline bool savePilotLayout(const std::string &path, const PilotLayout &l) {
    if (l.pilots.size() != (size_t)l.buckets * l.partitions || l.offsets.size() != (size_t)l.partitions + 1)
        return false;
    std::FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    const uint32_t head[4] = {l.partitions, l.buckets, l.partition_size, 0};
    bool ok = std::fwrite("PHBLAYT1", 1, 8, f) == 8 && std::fwrite(&l.n, 8, 1, f) == 1 &&
              std::fwrite(head, 4, 4, f) == 4 &&
              (l.pilots.empty() || std::fwrite(l.pilots.data(), 4, l.pilots.size(), f) == l.pilots.size()) &&
              std::fwrite(l.offsets.data(), 4, l.offsets.size(), f) == l.offsets.size();
    ok = std::fclose(f) == 0 && ok;
    return ok;
}

// False when the file is missing, has another magic, or its size does not match its header.
inline bool loadPilotLayout(const std::string &path, PilotLayout *l) {
    std::FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    char magic[8];
    uint32_t head[4];
    bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "PHBLAYT1", 8) == 0 &&
              std::fread(&l->n, 8, 1, f) == 1 && std::fread(head, 4, 4, f) == 4;
    if (ok) {
        l->partitions = head[0], l->buckets = head[1], l->partition_size = head[2];
        l->pilots.resize((size_t)l->buckets * l->partitions);
        l->offsets.resize((size_t)l->partitions + 1);
        ok = (l->pilots.empty() || std::fread(l->pilots.data(), 4, l->pilots.size(), f) == l->pilots.size()) &&
             std::fread(l->offsets.data(), 4, l->offsets.size(), f) == l->offsets.size() && std::fgetc(f) == EOF &&
             l->offsets[0] == 0 && l->offsets.back() == l->n;
    }
    std::fclose(f);
    return ok;
}

}  // namespace phobicgpu
