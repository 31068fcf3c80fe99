// qs_api.h — wraps every extern "C" entry point so that no C++ exception
// crosses the ABI: errors become status codes and the message is kept on the
// handle (or in a thread-local slot when there is no handle).
#pragma once
#include "qs_internal.h"

void qs_set_tls_error(const std::string& m);

#define QS_API_BEGIN try {
#define QS_API_END(h)                                                        \
  }                                                                          \
  catch (const qs_error& e) {                                                \
    if (h) (h)->err = e.what(); else qs_set_tls_error(e.what());             \
    return e.code;                                                           \
  }                                                                          \
  catch (const std::bad_alloc&) {                                            \
    if (h) (h)->err = "host allocation failed"; else qs_set_tls_error("host allocation failed"); \
    return QS_ERR_NOMEM;                                                     \
  }                                                                          \
  catch (const std::exception& e) {                                          \
    if (h) (h)->err = e.what(); else qs_set_tls_error(e.what());             \
    return QS_ERR_INVALID;                                                   \
  }                                                                          \
  return QS_OK;

#define QS_REQUIRE_HANDLE(h)                                                 \
  do { if (!(h)) { qs_set_tls_error("null handle"); return QS_ERR_INVALID; } } while (0)

inline void qs_check_state(const void* state, int n_qubits) {
  QS_CHECK_ARG(state != nullptr, "state pointer is null");
  QS_CHECK_ARG(((uintptr_t)state & 15u) == 0, "state must be 16-byte aligned");
  QS_CHECK_ARG(n_qubits >= 1 && n_qubits <= QS_MAX_QUBITS, "n_qubits out of range [1, 34]");
}
inline void qs_check_qubit(int q, int n_qubits, const char* what) {
  if (q < 0 || q >= n_qubits)
    throw qs_error(QS_ERR_INVALID, std::string(what) + " qubit index out of range");
}
