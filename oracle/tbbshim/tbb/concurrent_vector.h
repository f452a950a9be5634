// oneTBB-API stand-in (oracle test infrastructure only): included, unused by the reference path.
#pragma once
#include <vector>
namespace tbb { template <typename T> using concurrent_vector = std::vector<T>; }
