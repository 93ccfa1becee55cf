/* Pre-included (-include) when compiling the reference sources for the oracle:
 * claims the reference's config.h include guard so that the lattice size comes
 * from -DNS=<Nx> -DNT=<Nt> on the compiler command line instead of the
 * checked-in NS=NT=256.  Test infrastructure only. */
#define CONFIG_H
