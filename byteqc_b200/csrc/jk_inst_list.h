// generated: registration functions of the jk_inst_*.cu files
#pragma once
struct JKTables;
void jk_register_00(JKTables* T);
void jk_register_10(JKTables* T);
void jk_register_11(JKTables* T);
void jk_register_20(JKTables* T);
void jk_register_21(JKTables* T);
void jk_register_22(JKTables* T);
void jk_register_300(JKTables* T);
void jk_register_301(JKTables* T);
void jk_register_302(JKTables* T);
void jk_register_303(JKTables* T);
void jk_register_310(JKTables* T);
void jk_register_311(JKTables* T);
void jk_register_312(JKTables* T);
void jk_register_313(JKTables* T);
void jk_register_320(JKTables* T);
void jk_register_321(JKTables* T);
void jk_register_322(JKTables* T);
void jk_register_323(JKTables* T);
void jk_register_330(JKTables* T);
void jk_register_331(JKTables* T);
void jk_register_332(JKTables* T);
void jk_register_333(JKTables* T);
#define JK_REGISTER_ALL() \
jk_register_00(&g_tabs); \
jk_register_10(&g_tabs); \
jk_register_11(&g_tabs); \
jk_register_20(&g_tabs); \
jk_register_21(&g_tabs); \
jk_register_22(&g_tabs); \
jk_register_300(&g_tabs); \
jk_register_301(&g_tabs); \
jk_register_302(&g_tabs); \
jk_register_303(&g_tabs); \
jk_register_310(&g_tabs); \
jk_register_311(&g_tabs); \
jk_register_312(&g_tabs); \
jk_register_313(&g_tabs); \
jk_register_320(&g_tabs); \
jk_register_321(&g_tabs); \
jk_register_322(&g_tabs); \
jk_register_323(&g_tabs); \
jk_register_330(&g_tabs); \
jk_register_331(&g_tabs); \
jk_register_332(&g_tabs); \
jk_register_333(&g_tabs); \
    do {} while (0)
