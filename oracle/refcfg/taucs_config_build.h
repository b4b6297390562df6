/* Configuration header for compiling the unmodified reference sources as the
 * oracle.  The reference's own configurator would generate this file; these
 * few module switches are written by hand instead so that its build system is
 * never run.  Only the double-precision real instantiation is built, with the
 * ordering, supernodal LLT, unified-solver and support modules it needs. */
#define TAUCS_OSTYPE linux
#define TAUCS_VARIANT none
#define OSTYPE_linux
#define OSTYPE_VARIANT_none
#define TAUCS_CONFIG_DREAL
#define TAUCS_CONFIG_GENERIC_COMPLEX
#define TAUCS_CONFIG_TIMING
#define TAUCS_CONFIG_BASE
#define TAUCS_CONFIG_AMD
#define TAUCS_CONFIG_GENMMD
#define TAUCS_CONFIG_ORDERING
#define TAUCS_CONFIG_FACTOR
#define TAUCS_CONFIG_LLT
#define TAUCS_CONFIG_OOC_LLT
#define TAUCS_CONFIG_ADVANCED_MEMORY_OPS
#define TAUCS_CONFIG_VAIDYA
#define TAUCS_CONFIG_INCOMPLETE_CHOL
