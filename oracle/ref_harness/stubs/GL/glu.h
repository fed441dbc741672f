/* Empty stand-in: the reference includes OpenGL headers only for its display structs. */
