/* A plain C consumer of include/mdff_gpu.h, as a Fortran bind(c) or C host
   program sees it: compiled by gcc, linked against libmdff_gpu.so, it checks
   that the C compiler lays out every ABI struct with the sizes and field
   offsets the library was built with, and that the status strings resolve.
   Calls no function that needs a GPU.  Exit status 0 = layouts agree. */
#include <stddef.h>
#include <stdio.h>
#include <string.h>

#include "mdff_gpu.h"

static int check(const char* name, int which, size_t c_size) {
  int lib = mdff_gpu_struct_size(which);
  printf("%-16s C %6zu  library %6d\n", name, c_size, lib);
  return lib == (int)c_size ? 0 : 1;
}

int main(void) {
  int bad = 0;
  if (mdff_gpu_abi_version() != MDFF_ABI_VERSION) {
    printf("ABI version: header %d, library %d\n", MDFF_ABI_VERSION, mdff_gpu_abi_version());
    bad = 1;
  }
  bad |= check("mdff_params", 0, sizeof(mdff_params));
  bad |= check("mdff_result", 1, sizeof(mdff_result));
  bad |= check("mdff_stats", 2, sizeof(mdff_stats));
  bad |= check("mdff_batch_desc", 3, sizeof(mdff_batch_desc));
  bad |= check("mdff_batch_conf", 4, sizeof(mdff_batch_conf));
  /* the last fields of mdff_params close the struct with no trailing gap a
     Fortran mirror would miss */
  printf("offset rcut_wfc %zu, end %zu\n", offsetof(mdff_params, rcut_wfc), sizeof(mdff_params));
  if (offsetof(mdff_params, rcut_wfc) + sizeof(double) != sizeof(mdff_params)) bad = 1;
  for (int s = MDFF_OK; s <= MDFF_ERR_NOMEM; ++s)
    if (!mdff_gpu_strerror(s) || !strcmp(mdff_gpu_strerror(s), "unknown status")) bad = 1;
  printf(bad ? "layout mismatch\n" : "layouts agree\n");
  return bad;
}
