/*
 * Forced-include shim used ONLY to compile the reference's own CPU classes
 * (CaSim/*.cpp, read in place) into oracle/_ref/ with g++ on Linux.
 * It is test infrastructure: nothing in the product links it.
 *
 * Why each line exists:
 *  - `using std::abs;`  The reference calls unqualified abs(double) inside
 *    every GaussElimination (e.g. CaSim/DyadRD2DCPU.cpp:166-168). MSVC, the
 *    compiler the reference targets, resolves that to the floating overload;
 *    libstdc++ resolves it to int abs(int), which silently zeroes pivots
 *    below 1.0. Bringing std::abs into scope restores the MSVC meaning.
 *  - operator*(double, const json&)  CaSim/CytosolPool.cpp:104,112 multiply a
 *    double by a json value; with nlohmann 3.11 that is ambiguous between the
 *    built-in arithmetic candidates. A non-template exact match resolves it to
 *    the intended double product without editing the reference source.
 *  - #undef M_PI  CaSim/spline.h:40-41 redefines M_PI.
 */
#pragma once
#include <cmath>
#include <cstdlib>
#include <algorithm>
#include <vector>
#include <string>
#include <map>
#include <memory>
#include <fstream>
#include <iostream>
#include <functional>
#include <unordered_map>
#include <nlohmann/json.hpp>

using std::abs;

inline double operator*(double a, const nlohmann::json& b) { return a * b.get<double>(); }

#ifdef M_PI
#undef M_PI
#endif
