/* Stand-in for the compile_time_info.c that GALIC's prepare-config.perl
 * generates; lists the options in galicconfig.h.  CPU oracle only. */
#include <stdio.h>
void output_compile_time_options(void) { printf("        DOUBLEPRECISION=1\n        VER_1_1\n\n"); }
