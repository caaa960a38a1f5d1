/*
 * ORACLE — test infrastructure only.
 *
 * NDRange executor for the reference kernels compiled through clshim.h.
 * Work-group rows are spread over OpenMP threads; a thread runs the groups of
 * its row in ascending x and the work items of a group in local linear order.
 * Because pmhstereo_propagate_view only appends view candidates to pixels of
 * its own row (pmhstereo.cl:1064), this fixes the atomic_inc order to that of
 * a sequential executor.  Kernels that call barrier() run each work item as a
 * fiber (ucontext) that yields at the barrier.
 */
#ifndef PM_REF_EXEC_H
#define PM_REF_EXEC_H

#include <functional>

#include "clshim.h"

namespace clk {
void nd_range(int gw, int gh, int lw, int lh, bool barriers, const std::function<void()>& fn);
}

#endif
