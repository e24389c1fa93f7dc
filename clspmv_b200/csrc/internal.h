// Internal helpers shared by the host translation units of libclspmv_b200.
#pragma once

#include <stdarg.h>
#include "csp/clspmv.h"

namespace csp {

// Records a detail message for csp_last_error() on the calling thread and returns `code`.
int set_error(int code, const char* fmt, ...);
void clear_error();

int check_coo(const coo_matrix_if* m);
bool coo_is_sorted(const coo_matrix_if* m);
int ensure_sorted(coo_matrix_if* m);

}  // namespace csp
