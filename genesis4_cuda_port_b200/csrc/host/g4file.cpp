// g4file.cpp -- the host layer's output and dump files.
//
// Upstream GENESIS 1.3 v4 writes its records (rootname.out.h5), particle
// dumps (.par.h5) and field dumps (.fld.h5) with HDF5, which this build does
// not have.  The same datasets, under the same HDF5-style path names, go into
// one self-describing little-endian container per file ("G4DS" format):
//
//   bytes 0-7   magic "G4DS" 0 0 0 1 (format version 1)
//   u64         number of datasets
//   per dataset:
//     u32       name length, then the name ('/'-separated group path)
//     u32       element type (0 = float64, 1 = int64)
//     u32       rank, then rank x u64 dimensions (row-major, slowest first)
//     payload   product(dimensions) x 8 bytes
//
// Writers: the run's records (Diagnostic::val, Lattice tables), and the
// marker dumps of ControlCUDA::applyMarker (src/Core/ControlCUDA.cpp:131-146).
// Readers: the deck's &importbeam / &importfield, and g4h_file_* for callers.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <string>
#include <vector>

#include "g4file.h"
#include "g4h_internal.h"

namespace g4h {

namespace {
const char kMagic[8] = {'G', '4', 'D', 'S', 0, 0, 0, 1};
}

void DataFile::add(const std::string& name, std::vector<uint64_t> dims,
                   const std::vector<double>& data) {
  Dataset d;
  d.name = name;
  d.dims = std::move(dims);
  d.data = data;
  sets[name] = std::move(d);
}

void DataFile::add_scalar(const std::string& name, double v) { add(name, {1}, {v}); }

const Dataset* DataFile::find(const std::string& name) const {
  auto it = sets.find(name);
  return it == sets.end() ? nullptr : &it->second;
}

bool DataFile::write(const std::string& path) const {
  std::ofstream os(path, std::ios::binary | std::ios::trunc);
  if (!os) {
    set_error("cannot open " + path + " for writing");
    return false;
  }
  auto u32 = [&](uint32_t v) { os.write(reinterpret_cast<const char*>(&v), 4); };
  auto u64 = [&](uint64_t v) { os.write(reinterpret_cast<const char*>(&v), 8); };
  os.write(kMagic, 8);
  u64(sets.size());
  for (auto& [name, d] : sets) {
    u32((uint32_t)name.size());
    os.write(name.data(), (std::streamsize)name.size());
    u32(d.type);
    u32((uint32_t)d.dims.size());
    uint64_t n = 1;
    for (uint64_t v : d.dims) {
      u64(v);
      n *= v;
    }
    if (n != d.data.size()) {
      set_error("dataset " + name + ": dimensions do not match its data");
      return false;
    }
    os.write(reinterpret_cast<const char*>(d.data.data()), (std::streamsize)(8 * n));
  }
  if (!os) {
    set_error("write to " + path + " failed");
    return false;
  }
  return true;
}

bool DataFile::read(const std::string& path) {
  std::ifstream is(path, std::ios::binary);
  if (!is) {
    set_error("cannot open " + path);
    return false;
  }
  char magic[8];
  is.read(magic, 8);
  if (!is || std::memcmp(magic, kMagic, 8) != 0) {
    set_error(path + " is not a G4DS file");
    return false;
  }
  auto u32 = [&]() {
    uint32_t v = 0;
    is.read(reinterpret_cast<char*>(&v), 4);
    return v;
  };
  auto u64 = [&]() {
    uint64_t v = 0;
    is.read(reinterpret_cast<char*>(&v), 8);
    return v;
  };
  sets.clear();
  const uint64_t count = u64();
  for (uint64_t i = 0; i < count && is; ++i) {
    Dataset d;
    const uint32_t nl = u32();
    if (nl > 4096) break;
    d.name.resize(nl);
    is.read(&d.name[0], nl);
    d.type = u32();
    const uint32_t rank = u32();
    if (rank > 8) break;
    uint64_t n = 1;
    for (uint32_t k = 0; k < rank; ++k) {
      d.dims.push_back(u64());
      n *= d.dims.back();
    }
    if (n > (1ull << 36)) break;
    d.data.resize(n);
    is.read(reinterpret_cast<char*>(d.data.data()), (std::streamsize)(8 * n));
    sets[d.name] = std::move(d);
  }
  if (!is || sets.size() != count) {
    set_error(path + ": truncated or malformed G4DS file");
    return false;
  }
  return true;
}

std::string slice_group(int s) {
  char buf[32];
  std::snprintf(buf, sizeof buf, "slice%06d", s + 1);
  return buf;
}

}  // namespace g4h

using namespace g4h;

extern "C" {

int g4h_file_list(const char* path, char* buf, int buflen, int* needed) {
  if (!path) {
    set_error("g4h_file_list: null path");
    return G4B_ERR_ARG;
  }
  DataFile f;
  if (!f.read(path)) return G4B_ERR_ARG;
  std::string s;
  for (auto& kv : f.sets) s += kv.first + "\n";
  if (needed) *needed = (int)s.size() + 1;
  if (buf && buflen > 0) {
    const size_t n = std::min((size_t)buflen - 1, s.size());
    std::memcpy(buf, s.data(), n);
    buf[n] = 0;
  }
  return G4B_OK;
}

int g4h_file_read(const char* path, const char* name, double* out, int64_t capacity,
                  int64_t* length, int* rank, int64_t* dims) {
  if (!path || !name) {
    set_error("g4h_file_read: null argument");
    return G4B_ERR_ARG;
  }
  DataFile f;
  if (!f.read(path)) return G4B_ERR_ARG;
  const Dataset* d = f.find(name);
  if (!d) {
    set_error(std::string("g4h_file_read: no dataset ") + name + " in " + path);
    return G4B_ERR_ARG;
  }
  if (length) *length = (int64_t)d->data.size();
  if (rank) *rank = (int)d->dims.size();
  if (dims)
    for (size_t k = 0; k < d->dims.size() && k < 8; ++k) dims[k] = (int64_t)d->dims[k];
  if (out)
    std::memcpy(out, d->data.data(), 8 * (size_t)std::min<int64_t>(capacity, d->data.size()));
  return G4B_OK;
}

}  // extern "C"
