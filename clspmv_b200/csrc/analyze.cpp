// Cocktail analyzer (placeholder until the partitioner lands).
#include "csp/clspmv.h"
#include "internal.h"

extern "C" int csp_analyze_matrix(coo_matrix_if* coo, cocktail_iif* mat, const csp_analyze_opts* opts)
{
    (void)coo; (void)mat; (void)opts;
    return csp::set_error(CSP_EUNSUP, "analyzer not built yet");
}
