/* Stand-in for the CUDA runtime header: the host build of the reference gets its CUDA vocabulary from ref_shim.h. */
