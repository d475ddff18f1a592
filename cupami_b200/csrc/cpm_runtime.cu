// cupami_b200 runtime: the C ABI declared in include/cupami_b200.h.
//
// Host side of the vertical-bitset miner: device memory, database loading,
// the Eclat and Apriori drivers, and result ordering.  All arithmetic on
// transactions runs in the CUDA kernels included below; the host only plans
// (buffer sizes, class order) and moves counts and results.
#include "../../include/cupami_b200.h"
#include "common.cuh"
#include "k_basic.cuh"
#include "k_pairs.cuh"
#include "k_batch.cuh"
#include "k_gram_tc.cuh"
#include "k_deep.cuh"
#include "k_local.cuh"
#include "k_rows.cuh"
#include "k_apriori.cuh"
#include "k_periodic.cuh"
#include "k_costmodel.cuh"
#include "k_units.cuh"
#include "k_text.cuh"
#include <cub/device/device_radix_sort.cuh>

#include <cub/device/device_scan.cuh>
#include <thrust/iterator/transform_iterator.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>
#include <unordered_set>
#include <vector>
#include <map>
#include <memory>
#include <array>
#include <chrono>
#include <cstdlib>
#include <mutex>
#include <deque>
#include <cmath>

using namespace cpm;

#include "rt_context.inc"
#include "rt_database.inc"
#include "rt_pairs.inc"
#include "rt_deep.inc"
#include "rt_eclat.inc"
#include "rt_apriori.inc"
#include "rt_periodic.inc"
#include "rt_entry.inc"
#include "rt_results.inc"
#include "rt_kernel_api.inc"
#include "rt_costmodel.inc"
#include "rt_noalloc.inc"
#include "rt_text.inc"
#include "rt_labels.inc"
