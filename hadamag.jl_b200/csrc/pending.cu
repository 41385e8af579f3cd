// pending.cu -- entry points whose kernels are not in this build yet; each returns
// HM_ERR_ARG with a message instead of computing anything.
#include "hm_ctx.h"

extern "C" {
int hm_sre_grad(hm_ctx *c, const double *, int, double, double *, double *) {
  return c ? hm::set_err(c, HM_ERR_ARG, "hm_sre_grad: not available in this build") : HM_ERR_ARG;
}
int hm_mc_sre(hm_ctx *c, const double *, int, double, int, int, const uint64_t *, const double *, double *, double *,
              double *, double *, uint64_t *) {
  return c ? hm::set_err(c, HM_ERR_ARG, "hm_mc_sre: not available in this build") : HM_ERR_ARG;
}
int hm_mana_pure(hm_ctx *c, const double *, int, double *) {
  return c ? hm::set_err(c, HM_ERR_ARG, "hm_mana_pure: not available in this build") : HM_ERR_ARG;
}
int hm_mana_mixed(hm_ctx *c, const double *, int, double *) {
  return c ? hm::set_err(c, HM_ERR_ARG, "hm_mana_mixed: not available in this build") : HM_ERR_ARG;
}
int hm_sre_batched(hm_ctx *c, int, const double *const *, const int *, const double *, int, int, double *, double *) {
  return c ? hm::set_err(c, HM_ERR_ARG, "hm_sre_batched: not available in this build") : HM_ERR_ARG;
}
}
