// force_variants.cu -- the autotuner's table of force-kernel launch variants.
#include "force_impl.cuh"

namespace qgb
{
int force_variant_count() { return N_FORCE_VARIANTS; }
int batch_force_variant_count() { return N_BATCH_FORCE_VARIANTS; }
int force_variant_info_c(int variant, int* bs, int* minb, int* split, int* map)
{
  return force_variant_info(variant, bs, minb, split, map);
}
}  // namespace qgb
