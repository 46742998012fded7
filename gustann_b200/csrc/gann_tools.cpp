// Index-preparation helpers exported next to the search ABI.
#include <algorithm>
#include <cstdint>
#include <random>
#include <vector>

#include "gann_internal.h"

extern "C" {

/* Pivot-graph sample of bin/gen_small_file.cpp:12-25: the ids 0..num_data-1
 * shuffled by std::shuffle with std::mt19937(seed) (the reference uses 114514),
 * truncated to num_samp and sorted ascending. Written to out[num_samp]. */
int gann_sample_pivots(int64_t num_data, int64_t num_samp, uint32_t seed, int32_t* out) {
  if (num_data <= 0 || num_data > INT32_MAX || num_samp < 0 || num_samp > num_data || !out) return GANN_EINVAL;
  std::mt19937 gen(seed);
  std::vector<int> vec((size_t)num_data);
  for (int64_t i = 0; i < num_data; i++) vec[(size_t)i] = (int)i;
  std::shuffle(vec.begin(), vec.end(), gen);
  vec.resize((size_t)num_samp);
  std::sort(vec.begin(), vec.end());
  std::copy(vec.begin(), vec.end(), out);
  return GANN_OK;
}

}  // extern "C"
