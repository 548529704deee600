// Instantiations of the J/K launchers for one slice of the classes (one
// file per slice so the build compiles them in parallel).
#include "jk_launch.cuh"

void jk_register_11(JKTables* T) {
    JK_REG(1, 1, 0, 0)
    JK_REG(1, 1, 1, 0)
    JK_REG(1, 1, 1, 1)
}
