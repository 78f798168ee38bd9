// Binding that compiles the reference's own CPU scan, unmodified, from the
// reference checkout (src/torch/torch_scan_cpu.h:24-107).  Built by
// oracle/build_ref.py into oracle/_ref/; used only as the parity pin and the
// timed "reference" CPU baseline, never by the product.
#include "torch_scan_cpu.h"

#include <omp.h>

static int ref_max_threads() { return omp_get_max_threads(); }

PYBIND11_MODULE(tcuscan_ref_cpu, m) {
  m.def("run_scan_cpu", &tcuscan::run_scan_cpu, "reference run_scan_cpu");
  m.def("omp_max_threads", &ref_max_threads, "omp_get_max_threads()");
}
