// Test-infrastructure stand-in for libzmq's C header (not installed here); the
// reference engine includes it but uses only the C++ names from zmq.hpp.
#pragma once
#include "zmq.hpp"
