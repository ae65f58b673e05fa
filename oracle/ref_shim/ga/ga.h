/* TEST INFRASTRUCTURE ONLY.  Stand-in for Global Arrays' ga.h, which is not part of
 * the TAMM tree: just the types, enums and single-process queries that TAMM's
 * kernels/multiply.hpp include chain names (types.hpp, rmm_memory_pool.hpp). */
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

typedef int ga_nbhdl_t;
inline void NGA_NbWait(ga_nbhdl_t*) {}
inline int  GA_Nodeid() { return 0; }
inline int  GA_Cluster_nodeid() { return 0; }
inline int  GA_Cluster_nprocs(int) { return 1; }
inline int  GA_Initialized() { return 1; }
enum { C_FLOAT = 1, C_DBL, C_SCPL, C_DCPL, C_INT, C_LONG };
