// Umbrella header of the B200 PHOBIC engine's C++ layer; the counterpart of the
// reference's include/phobic_gpu_mphf.hpp:1-22.  Code written against the
// reference compiles against this header: MPHFconfig, MPHFbuilder, MPHF and the
// encoders keep their names; MPHFbuilder::build runs on the GPU through the C ABI.
//
//   #include "phobic_gpu_mphf.hpp"
//   phobicgpu::MPHFbuilder builder(phobicgpu::MPHFconfig(7.0, 2500));
//   phobicgpu::FastQueryMphf f;
//   builder.build(keys, f);          // keys: std::vector<uint64_t | std::string | ...>
//   uint32_t slot = f(keys[0]);      // in [0, n)
//
// Compile with -I<repo>/include -I<repo>/phobic-gpu_b200/cpp [-fopenmp], link
// -L<repo>/phobic-gpu_b200/lib -lphobic_b200.
#pragma once

#include "phobicB200/builder.hpp"
#include "phobicB200/config.hpp"
#include "phobicB200/encoders.hpp"
#include "phobicB200/layout.hpp"
#include "phobicB200/mphf.hpp"

namespace phobicgpu {

typedef MPHF<interleaved_encoder<compact>, diff_partition_encoder<compact>, xxhash> FastQueryMphf;
typedef MPHF<interleaved_encoder<rice>, diff_partition_encoder<compact>, xxhash> SmallSpaceMphf;

}  // namespace phobicgpu
