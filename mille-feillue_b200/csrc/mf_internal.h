// Internal declarations shared by the host C++ and CUDA sources of libmf.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "mf.h"

struct mf_matrix {
    int n = 0, ncols = 0;
    std::vector<int> row_ptr, col_idx;
    std::vector<double> val;
    std::vector<double> b, xstar;  // optional right-hand side / exact solution
};

namespace mf {

// Deterministic uniform draws in [0,1) with 53 random bits from mt19937_64.
struct Rng;

// Tile constants (BLOCK_SIZE of the reference, Performance-Comparison/common.h:47-50).
constexpr int TILE = 16;

void set_last_error(const std::string &msg);
const std::string &last_error();

}  // namespace mf
