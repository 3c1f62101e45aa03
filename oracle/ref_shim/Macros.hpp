// Minimal stand-in for LvArray's Macros.hpp: only the error, logging and stringizing macros that the
// reference's hot-path sources use.  Part of the oracle's reference build (test infrastructure).
#pragma once

#include <sstream>
#include <stdexcept>
#include <string>

#define STRINGIZE_NX(A) #A
#define STRINGIZE(A) STRINGIZE_NX(A)

#define LVARRAY_UNUSED_ARG(X)
#define LVARRAY_UNUSED_VARIABLE(X) ((void) (X))
#define LVARRAY_HOST_DEVICE
#define LVARRAY_DEVICE

#define LVARRAY_ERROR_IF(EXP, MSG)                                                                    \
  do {                                                                                                \
    if (EXP) {                                                                                        \
      std::ostringstream __oss;                                                                       \
      __oss << __FILE__ << ":" << __LINE__ << ": " << STRINGIZE(EXP) << ": " << MSG;                \
      throw std::runtime_error(__oss.str());                                                          \
    }                                                                                                 \
  } while (false)

#define LVARRAY_ERROR(MSG) LVARRAY_ERROR_IF(true, MSG)
#define LVARRAY_THROW_IF(EXP, MSG, TYPE)                                                              \
  do {                                                                                                \
    if (EXP) {                                                                                        \
      std::ostringstream __oss;                                                                       \
      __oss << __FILE__ << ":" << __LINE__ << ": " << MSG;                                            \
      throw TYPE(__oss.str());                                                                        \
    }                                                                                                 \
  } while (false)
#define LVARRAY_ERROR_IF_OP_MSG(L, OP, R, MSG) LVARRAY_ERROR_IF((L) OP (R), (L) << " " STRINGIZE(OP) " " << (R) << " " << MSG)
#define LVARRAY_ERROR_IF_EQ(L, R) LVARRAY_ERROR_IF_OP_MSG(L, ==, R, "")
#define LVARRAY_ERROR_IF_NE(L, R) LVARRAY_ERROR_IF_OP_MSG(L, !=, R, "")
#define LVARRAY_ERROR_IF_GT(L, R) LVARRAY_ERROR_IF_OP_MSG(L, >, R, "")
#define LVARRAY_ERROR_IF_GE(L, R) LVARRAY_ERROR_IF_OP_MSG(L, >=, R, "")
#define LVARRAY_ERROR_IF_LT(L, R) LVARRAY_ERROR_IF_OP_MSG(L, <, R, "")
#define LVARRAY_ERROR_IF_LE(L, R) LVARRAY_ERROR_IF_OP_MSG(L, <=, R, "")
#define LVARRAY_ERROR_IF_NE_MSG(L, R, MSG) LVARRAY_ERROR_IF_OP_MSG(L, !=, R, MSG)
#define LVARRAY_ERROR_IF_GT_MSG(L, R, MSG) LVARRAY_ERROR_IF_OP_MSG(L, >, R, MSG)
#define LVARRAY_ERROR_IF_LT_MSG(L, R, MSG) LVARRAY_ERROR_IF_OP_MSG(L, <, R, MSG)
#define LVARRAY_ASSERT(EXP) LVARRAY_ERROR_IF(!(EXP), "")
#define LVARRAY_ASSERT_EQ(L, R) LVARRAY_ERROR_IF_NE(L, R)
#define LVARRAY_LOG(MSG) ((void) 0)
#define LVARRAY_LOG_VAR(VAR) ((void) 0)
#define LVARRAY_WARNING(MSG) ((void) 0)
#define LVARRAY_WARNING_IF(EXP, MSG) ((void) 0)
