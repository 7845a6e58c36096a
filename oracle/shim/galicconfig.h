/* Build configuration of the CPU oracle's copy of GALIC: the reference's
 * default Config.sh.template options (DOUBLEPRECISION=1, VER_1_1). */
#define DOUBLEPRECISION 1
#define VER_1_1
