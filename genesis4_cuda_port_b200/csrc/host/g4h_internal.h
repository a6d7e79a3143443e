// g4h_internal.h -- private helpers of the C++ host layer.
#pragma once

#include <cstdint>
#include <string>

namespace g4h {

void set_error(const std::string& m);
const char* last_error();

double radical_inverse(uint64_t i, unsigned base);
double inv_normal(double p);

struct Rng {
  uint64_t s;
  double uniform();
  double normal();
};

}  // namespace g4h
