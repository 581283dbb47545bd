/* empty stand-in: the reference includes <mkl.h> but calls nothing from it on the search path */
