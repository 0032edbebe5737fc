// Exception-to-status guard shared by the C ABI entry points: every entry
// point body runs between API_BEGIN and API_END, which turn a thrown
// aifmm::Error into its status code (and the last-error message) and any
// other exception into AIFMM_EINVAL / AIFMM_ENOMEM.
#pragma once
#include <new>
#include <stdexcept>

#include "common.cuh"

#define API_BEGIN try {
#define API_END                                        \
  }                                                    \
  catch (const ::aifmm::Error& e) {                    \
    ::aifmm::set_last_error(e.what());                 \
    return e.code;                                     \
  }                                                    \
  catch (const std::bad_alloc&) {                      \
    ::aifmm::set_last_error("host allocation failed"); \
    return AIFMM_ENOMEM;                               \
  }                                                    \
  catch (const std::exception& e) {                    \
    ::aifmm::set_last_error(e.what());                 \
    return AIFMM_EINVAL;                               \
  }                                                    \
  return AIFMM_OK;
