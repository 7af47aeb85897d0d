// The benchmark programs' entry point (nvbench::main).
#define NVBENCH_MAIN_HERE
#include <nvbench/nvbench.cuh>
