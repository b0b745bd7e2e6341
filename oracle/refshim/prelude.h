// Force-included ahead of the reference's own sources when oracle/Makefile
// builds them into oracle/_ref (test infrastructure).  It papers over the
// snapshot's source rot without touching the sources:
//  * FluidSim/include/FluidSim/fluid-sim.h names `core::` where Core declares
//    `sim::core` (Core/include/Core/core.h:12): `sim` is made an inline
//    namespace, so `core::X` and `sim::core::X` name the same entity;
//  * spatify::NeighbourSearcher (FluidSim/include/FluidSim/cpu/sdf.h:228) is
//    not declared anywhere: it is taken to be ParticleNeighbourSearcher
//    (Spatify/include/Spatify/ns-util.h:15-19), the only neighbour searcher;
//  * the ERROR macro is undefined in the tree: it prints and aborts;
//  * Spatify's parallel.h only compiles with USE_TBB, which refshim/tbb serves
//    serially.
#pragma once
#include <algorithm>
#include <array>
#include <cassert>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <format>
#include <fstream>
#include <functional>
#include <iostream>
#include <map>
#include <memory>
#include <numeric>
#include <optional>
#include <random>
#include <source_location>
#include <span>
#include <sstream>
#include <string>
#include <tuple>
#include <type_traits>
#include <unordered_map>
#include <utility>
#include <vector>
#define USE_TBB 1
#define ERROR(msg) (std::fprintf(stderr, "%s\n", msg), std::abort())
inline namespace sim { namespace core {} }
namespace spatify {
template <typename T, int Dim> class ParticleNeighbourSearcher;
template <typename T, int Dim> using NeighbourSearcher = ParticleNeighbourSearcher<T, Dim>;
}
