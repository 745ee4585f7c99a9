// Part of the Taskflow-API shim: the reference includes this header; all of
// the subset it uses lives in taskflow.hpp.
#pragma once
#include "../taskflow.hpp"
