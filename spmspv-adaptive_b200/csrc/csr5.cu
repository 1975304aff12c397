// CSR5 SpMV / SpMSpV (placeholder until the tile format lands).
#include "engine.h"
using namespace spmx;

extern "C" int spmx_set_sigma(spmx_handle_t h, int sigma) {
  if (!h) return set_error(SPMX_ERR_INVALID_VALUE, "NULL handle");
  h->sigma = sigma;
  return SPMX_SUCCESS;
}
extern "C" int spmx_csr5_preprocess(spmx_handle_t h) {
  if (!h) return set_error(SPMX_ERR_INVALID_VALUE, "NULL handle");
  return set_error(SPMX_ERR_NOT_READY, "CSR5 is not built yet");
}
extern "C" int spmx_csr5_postprocess(spmx_handle_t h) {
  if (!h) return set_error(SPMX_ERR_INVALID_VALUE, "NULL handle");
  return SPMX_SUCCESS;
}
int csr5_spmv_impl(spmx_handle_t h, float, float*, bool) {
  return set_error(SPMX_ERR_NOT_READY, "CSR5 is not built yet");
}
int csc_bucket_impl(spmx_handle_t h, float, float*, int*, float*, int*, int) {
  return set_error(SPMX_ERR_NOT_READY, "bucket SpMSpV is not built yet");
}
