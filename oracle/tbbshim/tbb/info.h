// oneTBB-API stand-in (oracle test infrastructure only; see detail_pool.h).
#pragma once
#include <vector>
namespace tbb { namespace info { inline std::vector<int> numa_nodes() { return {0}; } } }
