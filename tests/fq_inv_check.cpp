// Host driver for tests/test_fq_inv.py: runs the library's branch-free
// divstep Fq inversion (zk_gpu_b200/csrc/fq_inv.cuh, the same code the MSM kernels
// run) on values read from stdin (hex, one per line) and prints the inverses.
#include <cstdint>
#include <cstdio>
#define __host__
#define __device__
#include "../zk_gpu_b200/csrc/fq_inv.cuh"

int main() {
  char line[128];
  while (std::fgets(line, sizeof(line), stdin)) {
    uint32_t a[8] = {0}, r[8];
    // 64 hex digits, most significant first
    for (int i = 0; i < 8; i++) std::sscanf(line + 8 * (7 - i), "%8x", &a[i]);
    zk::fq_inv_divsteps(r, a);
    for (int i = 7; i >= 0; i--) std::printf("%08x", r[i]);
    std::printf("\n");
  }
  return 0;
}
