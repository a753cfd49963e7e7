/* TEST INFRASTRUCTURE ONLY: the FP64 instantiation of riptide_oracle.c (ora64_* symbols),
 * used to state each output's error against FP64. */
#define ORA_T double
#define ORA(name) ora64_##name
#include "riptide_oracle.c"
