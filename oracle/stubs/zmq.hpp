// Test-infrastructure stand-in for cppzmq's zmq.hpp (libzmq headers are not installed
// here). protocol.h needs <format>/<cstring>/<stdexcept> from it; the reference engine
// (src/engine.cpp) needs zmq::socket_t::send and zmq::buffer. This socket records the
// frames it is given instead of sending them, so that the engine can be driven in-process.
#pragma once
#include <cstdint>
#include <cstring>
#include <format>
#include <stdexcept>
#include <vector>

namespace zmq
{
struct const_buffer
{
    const void* data;
    size_t size;
};

inline const_buffer buffer(const std::vector<uint8_t>& v)
{
    return const_buffer{v.data(), v.size()};
}

struct socket_t
{
    std::vector<std::vector<uint8_t>>* frames = nullptr;
    void send(const_buffer b)
    {
        if (frames)
            frames->emplace_back((const uint8_t*)b.data, (const uint8_t*)b.data + b.size);
    }
};
} // namespace zmq
