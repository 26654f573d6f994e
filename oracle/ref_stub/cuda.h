/* Stand-in for the CUDA driver header: the host build of the reference gets its CUDA vocabulary from ref_shim.h. */
