/* Empty build configuration for compiling reference task sources against the
 * CPU shims in this directory (test infrastructure only). */
