// generated: registration functions of the jk_inst_*.cu files
#pragma once
void jk_register_00(jk_launch_fn* tab64, jk_launch_fn* tab32);
void jk_register_10(jk_launch_fn* tab64, jk_launch_fn* tab32);
void jk_register_11(jk_launch_fn* tab64, jk_launch_fn* tab32);
void jk_register_20(jk_launch_fn* tab64, jk_launch_fn* tab32);
void jk_register_21(jk_launch_fn* tab64, jk_launch_fn* tab32);
void jk_register_22(jk_launch_fn* tab64, jk_launch_fn* tab32);
void jk_register_300(jk_launch_fn* tab64, jk_launch_fn* tab32);
void jk_register_301(jk_launch_fn* tab64, jk_launch_fn* tab32);
void jk_register_302(jk_launch_fn* tab64, jk_launch_fn* tab32);
void jk_register_303(jk_launch_fn* tab64, jk_launch_fn* tab32);
void jk_register_310(jk_launch_fn* tab64, jk_launch_fn* tab32);
void jk_register_311(jk_launch_fn* tab64, jk_launch_fn* tab32);
void jk_register_312(jk_launch_fn* tab64, jk_launch_fn* tab32);
void jk_register_313(jk_launch_fn* tab64, jk_launch_fn* tab32);
void jk_register_320(jk_launch_fn* tab64, jk_launch_fn* tab32);
void jk_register_321(jk_launch_fn* tab64, jk_launch_fn* tab32);
void jk_register_322(jk_launch_fn* tab64, jk_launch_fn* tab32);
void jk_register_323(jk_launch_fn* tab64, jk_launch_fn* tab32);
void jk_register_330(jk_launch_fn* tab64, jk_launch_fn* tab32);
void jk_register_331(jk_launch_fn* tab64, jk_launch_fn* tab32);
void jk_register_332(jk_launch_fn* tab64, jk_launch_fn* tab32);
void jk_register_333(jk_launch_fn* tab64, jk_launch_fn* tab32);
#define JK_REGISTER_ALL() \
jk_register_00(g_tab64, g_tab32); \
jk_register_10(g_tab64, g_tab32); \
jk_register_11(g_tab64, g_tab32); \
jk_register_20(g_tab64, g_tab32); \
jk_register_21(g_tab64, g_tab32); \
jk_register_22(g_tab64, g_tab32); \
jk_register_300(g_tab64, g_tab32); \
jk_register_301(g_tab64, g_tab32); \
jk_register_302(g_tab64, g_tab32); \
jk_register_303(g_tab64, g_tab32); \
jk_register_310(g_tab64, g_tab32); \
jk_register_311(g_tab64, g_tab32); \
jk_register_312(g_tab64, g_tab32); \
jk_register_313(g_tab64, g_tab32); \
jk_register_320(g_tab64, g_tab32); \
jk_register_321(g_tab64, g_tab32); \
jk_register_322(g_tab64, g_tab32); \
jk_register_323(g_tab64, g_tab32); \
jk_register_330(g_tab64, g_tab32); \
jk_register_331(g_tab64, g_tab32); \
jk_register_332(g_tab64, g_tab32); \
jk_register_333(g_tab64, g_tab32); \
    do {} while (0)
