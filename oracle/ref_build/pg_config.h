/*
 * Minimal stand-in for the configure-generated pg_config.h, written by hand
 * for the oracle harness so that the reference's gpuqo sources compile
 * without running the reference's build system.
 *
 * Only the macros the gpuqo sources read are defined:
 *   BLCKSZ           - page size used by page_size() in the cost model
 *                      (src/backend/optimizer/gpuqo/gpuqo_cost_postgres.cuh:838)
 *   MAXIMUM_ALIGNOF  - MAXALIGN() in the hash-join sizing
 *                      (src/backend/optimizer/gpuqo/gpuqo_cost_postgres.cuh:31)
 * USE_ASSERT_CHECKING is left undefined (release build, as the reference's
 * benchmark configuration).
 *
 * This file is test infrastructure: only the oracle harness uses it.
 */
#ifndef ORACLE_PG_CONFIG_H
#define ORACLE_PG_CONFIG_H

#define BLCKSZ 8192
#define MAXIMUM_ALIGNOF 8

#endif
