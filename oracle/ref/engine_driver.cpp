// TEST INFRASTRUCTURE. Drives the reference's own simulation engine (src/engine.cpp,
// unchanged) with the controllers of drone-race_b200/adapter (the drop-in for
// include/controllers.h) for one closed-loop episode, in-process: the three header
// frames the Python front-end would send (python-src/protocol.py:225-229) go in, the
// frames the engine sends back (MSG_STATE / MSG_EVENT / MSG_DONE) come out. Mirrors
// runEngine (src/main.cpp:9-44) without the ZMQ transport.
#include "config.h"
#include "engine.h"

#include <cstring>
#include <fcntl.h>
#include <iostream>
#include <unistd.h>

extern "C" int engine_run_episode(const void* envF, size_t envN, const void* contF, size_t contN, const void* stF, size_t stN, int maxSteps, uint8_t* out,
                                  size_t outCap, size_t* outLen, int* nFrames, int quiet)
{
    int saved = -1;
    if (quiet)
    {
        std::cout.flush();
        fflush(stdout);
        saved = dup(1);
        int fd = open("/dev/null", O_WRONLY);
        dup2(fd, 1);
        close(fd);
    }
    int rc = 0;
    try
    {
        auto [envConfig, seed, trueTheta] = Env::unpackEnvConfig(envF, envN);
        AnyControllerConfig contConfig = loadControllerConfig(contF, contN);
        SimState init = Env::unpackSimState(stF, stN, envConfig);
        std::vector<std::vector<uint8_t>> frames;
        {
            SimulationEngine engine(envConfig, contConfig, init, seed, trueTheta);
            zmq::socket_t sock;
            sock.frames = &frames;
            engine.run(maxSteps, sock);
        }
        size_t off = 0;
        for (auto& f : frames)
        {
            if (off + 4 + f.size() > outCap)
            {
                rc = 2;
                break;
            }
            uint32_t n = (uint32_t)f.size();
            std::memcpy(out + off, &n, 4);
            std::memcpy(out + off + 4, f.data(), f.size());
            off += 4 + f.size();
        }
        *outLen = off;
        *nFrames = (int)frames.size();
    }
    catch (const std::exception& e)
    {
        std::cerr << "engine episode failed: " << e.what() << "\n";
        rc = 1;
    }
    if (quiet)
    {
        std::cout.flush();
        fflush(stdout);
        dup2(saved, 1);
        close(saved);
    }
    return rc;
}
