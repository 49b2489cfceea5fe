// sobol_tables_decl.h -- host accessor of the compiled-in Sobol tables' checksum (render.cu).
#pragma once
const char* pb2_sobol_table_sha256();
