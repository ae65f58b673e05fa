// Status-code wrapping shared by the extern "C" entry points: library exceptions
// become a status code plus tb_last_error(); nothing is thrown across the boundary.
#pragma once

#include "tb_internal.hpp"

#include <new>

#define TB_API_BEGIN try {
#define TB_API_END                                                                      \
  }                                                                                     \
  catch(const tb::Error& e) {                                                           \
    tb::set_last_error(e.what());                                                       \
    return e.code;                                                                      \
  }                                                                                     \
  catch(const std::bad_alloc&) {                                                        \
    tb::set_last_error("host allocation failed");                                       \
    return TB_ERR_NO_MEMORY;                                                            \
  }                                                                                     \
  catch(const std::exception& e) {                                                      \
    tb::set_last_error(e.what());                                                       \
    return TB_ERR_INVALID;                                                              \
  }                                                                                     \
  return TB_OK;

