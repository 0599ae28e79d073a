/* Empty stand-in for boost/preprocessor/repetition/repeat.hpp.
 * include/globals.hpp includes it unconditionally but only uses BOOST_PP_REPEAT
 * when FIXED_K is undefined; ref.mk defines FIXED_K, so nothing from it is used. */
