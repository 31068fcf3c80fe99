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

// Makes `dev` the calling thread's current device for the rest of the scope
// and restores the previous one at its end, so a handle's work always goes to
// its own device whatever device the caller had current.
struct qs_device_guard {
  int prev = -1;
  explicit qs_device_guard(int dev) {
    int cur = 0;
    if (cudaGetDevice(&cur) == cudaSuccess && cur != dev && cudaSetDevice(dev) == cudaSuccess) prev = cur;
  }
  ~qs_device_guard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
  qs_device_guard(const qs_device_guard&) = delete;
  qs_device_guard& operator=(const qs_device_guard&) = delete;
};

// First statement of every entry point that takes a handle: rejects a null
// handle and selects the handle's device until the call returns.
#define QS_REQUIRE_HANDLE(h)                                                 \
  if (!(h)) {                                                                \
    qs_set_tls_error("null handle");                                         \
    return QS_ERR_INVALID;                                                   \
  }                                                                          \
  const qs_device_guard qs_device_guard_((h)->device)

inline void qs_check_state(const void* state, int n_qubits) {
  QS_CHECK_ARG(state != nullptr, "state pointer is null");
  QS_CHECK_ARG(((uintptr_t)state & 15u) == 0, "state must be 16-byte aligned");
  QS_CHECK_ARG(n_qubits >= 1 && n_qubits <= QS_MAX_QUBITS, "n_qubits out of range [1, 34]");
}
inline void qs_check_qubit(int q, int n_qubits, const char* what) {
  if (q < 0 || q >= n_qubits)
    throw qs_error(QS_ERR_INVALID, std::string(what) + " qubit index out of range");
}
