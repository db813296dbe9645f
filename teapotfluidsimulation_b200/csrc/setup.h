#pragma once

#include <cstdio>
#include <vector>

#include "common.cuh"

namespace pl {

struct HostInit {
  Geo geo;
  double fill_height;
  std::vector<double> x, y, z;
  std::vector<uint8_t> origin;
  int band_counts[3];
};

int host_construct(const pl_config& cfg, HostInit* out, char* err, size_t errlen);

}  // namespace pl
