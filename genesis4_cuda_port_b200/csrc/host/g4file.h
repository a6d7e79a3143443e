// g4file.h -- G4DS dataset files (the host layer's stand-in for the upstream
// HDF5 output, particle-dump and field-dump files; format in g4file.cpp).
#pragma once

#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include "g4h.h"

namespace g4h {

struct Dataset {
  std::string name;
  uint32_t type = 0;  // 0 = float64
  std::vector<uint64_t> dims;
  std::vector<double> data;
};

struct DataFile {
  std::map<std::string, Dataset> sets;
  void add(const std::string& name, std::vector<uint64_t> dims, const std::vector<double>& data);
  void add_scalar(const std::string& name, double v);
  const Dataset* find(const std::string& name) const;
  bool write(const std::string& path) const;
  bool read(const std::string& path);
};

// "slice000001" for slice 0: the per-slice group names of upstream's dumps.
std::string slice_group(int s);

}  // namespace g4h
