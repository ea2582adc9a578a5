/* Test-only: include/neo_fft_b200.h used from plain C (C99, warnings as errors) and linked
 * against the library, calling the entry points that need no GPU: the ABI version, the config
 * defaults and the static scratch capacity. Prints the values for the caller to compare. */
#include <stdio.h>

#include "neo_fft_b200.h"

int main(void) {
  nf_fft3d_config f;
  nf_dft_config d;
  nf_fft3d_config_default(&f);
  nf_dft_config_default(&d);
  printf("%d %d %d %d %d %zu\n", nf_abi_version(), f.bw, f.bt, d.block, d.overlap,
         nf_dft_backward_static_capacity());
  return 0;
}
