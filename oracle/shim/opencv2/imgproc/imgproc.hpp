// TEST INFRASTRUCTURE ONLY.  See ../opencv.hpp (the project's OpenCV stand-in).
#pragma once
#include "../opencv.hpp"
