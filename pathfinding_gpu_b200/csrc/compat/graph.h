// graph.h (standalone builds) - the CSR graph type that include/gpu_sssp.h expects.
//
// Applications written against the reference keep using their own graph.h
// (the reference's include/graph.h, whose CSRGraph has these same fields);
// this header is for C++ programs that use the engine without the reference.
// Fields and meaning follow the reference's CSRGraph (include/graph.h:31-48):
// rows sorted by (w, dst), weights >= 1, optional planar coordinates and the
// admissible heuristic scale hScale.
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

using u8 = uint8_t;
using u32 = uint32_t;
using u64 = uint64_t;
using i64 = int64_t;

constexpr u32 INF_DIST = 0xFFFFFFFFu;
constexpr u32 NO_PARENT = 0xFFFFFFFFu;

struct CSRGraph {
    std::string name;
    u32 n = 0;
    u32 m = 0;
    std::vector<u32> row_offsets;  // n + 1
    std::vector<u32> col_indices;  // m
    std::vector<u32> weights;      // m
    std::vector<double> x, y;      // optional coordinates (A*)
    double hScale = 0.0;
    u32 minW = 0, maxW = 0, maxDeg = 0;
    double avgW = 0.0, avgDeg = 0.0;

    bool hasCoords() const { return !x.empty(); }
    u32 degree(u32 u) const { return row_offsets[u + 1] - row_offsets[u]; }
    size_t bytesCSR() const { return (size_t)(n + 1) * 4 + (size_t)m * 8; }
};
