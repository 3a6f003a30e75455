/*
 * The oracle's CPU restatement of the reference solver's hot path (TEST
 * INFRASTRUCTURE ONLY).  Instantiates simple_oracle_impl.h in FP64 (orc64_*,
 * the reference promoted to double, the parity reference) and FP32
 * (orc32_*, the reference as shipped).  Loaded by oracle/restatement.py via
 * ctypes; only tests, the smoke check and the CPU-baseline leg of bench.py use it.
 */
#include <math.h>
#include <stdlib.h>

#define REAL double
#define PREFIX orc64_
#include "simple_oracle_impl.h"
#undef REAL
#undef PREFIX

#define REAL float
#define PREFIX orc32_
#include "simple_oracle_impl.h"
#undef REAL
#undef PREFIX
