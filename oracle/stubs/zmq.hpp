// Minimal stand-in for cppzmq's zmq.hpp, used only to compile the reference's
// model headers (protocol.h includes zmq.hpp for <format>/<cstring>/<stdexcept>).
#pragma once
#include <cstring>
#include <format>
#include <stdexcept>
