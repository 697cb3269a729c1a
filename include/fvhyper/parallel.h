/*
 * fvhyper/parallel.h — process pool of the fvhyper API, B200 build.
 *
 * Same class and members as the reference (fvhyper/parallel.h:24-33), so a
 * user main() that constructs `fvhyper::mpi_wrapper pool;` and returns
 * `pool.exit()` compiles unchanged.  The B200 build runs one process per GPU
 * without MPI: rank = 0 and size = 1 (the MPI partition and halo exchange
 * are not part of the device path).
 */
#pragma once

namespace fvhyper {

class mpi_wrapper {
public:
    int rank;
    int size;

    mpi_wrapper();

    int exit();
};

}  // namespace fvhyper
