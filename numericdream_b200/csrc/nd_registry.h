// Formula registry shared by the generated table and the runtime.
#pragma once

#include <stdint.h>

#include "nd_kernels.cuh"

namespace nd {

struct ParamEntry {
  const char* name;
  float min_value, max_value, default_value;
  int integral;
};

// One build-time translated formula plugin.
struct FormulaEntry {
  const char* name;        // file stem
  uint64_t source_hash;    // FNV-1a 64 of the exact source bytes
  int nparams;
  ParamEntry params[ND_MAX_PARAMS];
  KernelTable (*kernels)();
  int32_t (*iterations)(const float* params);  // de_iterations(p) on the host
};

// A set of formulas compiled into one kernel (mixed-formula batches).
struct GroupEntry {
  const char* name;
  int count;
  int members[16];
  KernelTable (*kernels)();
};

}  // namespace nd

extern const nd::FormulaEntry nd_formula_entries[];
extern const int nd_formula_entry_count;

// Every formula the library knows: the build-time table (ids 0 .. nd_formula_entry_count
// - 1), then the formulas nd_formula_register compiled at run time.  nd_formula_at
// returns nullptr for an id out of range.
const nd::FormulaEntry* nd_formula_at(int id);
int nd_formula_total();
extern const nd::GroupEntry nd_group_entries[];
extern const int nd_group_entry_count;
