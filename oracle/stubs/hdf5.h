/* empty stand-in: the oracle build compiles no file-format I/O */
