// Shim: the reference only queries NUMA topology for core pinning helpers.
#pragma once
inline int numa_num_configured_cpus() { return 1; }
inline int numa_node_of_cpu(int) { return 0; }
