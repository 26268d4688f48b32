// Runs the reference's own main() (src/main.cpp, compiled unmodified with
// -Dmain=r3d_reference_main) on thread-ranks of the MPI stand-in (mpi_shim/): R3D_NRANKS ranks
// (default 2), each a host thread with its own copy of argv.  Test infrastructure: it lets the
// reference driver - with its --backend gpu branch bound to the B200 library through
// rast-3dmhd_b200/refbind/gpu_shim.cpp - run where no MPI library exists.  The exit status is
// the largest of the ranks' return values (1 for a rank that aborted).
#include <cstdio>
#include <cstdlib>
#include <exception>
#include <string>
#include <thread>
#include <vector>

#include "mpi.h"

int r3d_reference_main(int argc, char** argv);

int main(int argc, char** argv) {
    const char* env = getenv("R3D_NRANKS");
    const int n = env ? atoi(env) : 2;
    if (n < 1) {
        fprintf(stderr, "R3D_NRANKS must be >= 1\n");
        return 2;
    }
    r3d_shim_world_init(n);
    std::vector<int> rc(n, 0);
    std::vector<std::thread> th;
    for (int r = 0; r < n; ++r)
        th.emplace_back([&, r] {
            std::vector<std::string> args(argv, argv + argc);
            std::vector<char*> av;
            for (auto& a : args) av.push_back(&a[0]);
            av.push_back(nullptr);
            r3d_shim_bind_rank(r);
            try {
                rc[r] = r3d_reference_main(argc, av.data());
            } catch (const std::exception& e) {
                fprintf(stderr, "rank %d: %s\n", r, e.what());
                rc[r] = 1;
            }
        });
    for (auto& t : th) t.join();
    int worst = 0;
    for (int v : rc) worst = v > worst ? v : worst;
    return worst;
}
