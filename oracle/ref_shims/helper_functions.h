/* Empty stand-in for the CUDA-samples header named in include/FAME_CUDA.h:8. */
