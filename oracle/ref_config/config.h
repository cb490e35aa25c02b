/* Stand-in for the autoconf-generated config.h that the reference's
 * include/thread.h pulls in.  Every feature switch the oracle build needs is
 * passed on the compiler command line by oracle/Makefile, so this header is
 * intentionally empty.  It is test infrastructure, not product code. */
