// Project-written single-process stand-in (see detail/one_process.hpp).  Test infrastructure only.
#ifndef RBK_SHIM_YAMPI_STATUS_HPP
#define RBK_SHIM_YAMPI_STATUS_HPP
#include "detail/one_process.hpp"
#endif
