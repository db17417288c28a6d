/* TEST INFRASTRUCTURE ONLY.  Empty stand-in for the MSVC <intrin.h> that the
 * reference's vecmath.h includes; nothing from it is used by the DiTO code. */
