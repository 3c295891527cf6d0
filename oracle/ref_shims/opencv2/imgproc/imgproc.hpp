/* Build shim; see opencv2/opencv.hpp.  Test infrastructure only. */
#pragma once
#include "../opencv.hpp"
