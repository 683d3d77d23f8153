/* A minimal NVTX injection tool for the trace test: counts the ASCII range pushes and the
 * pops it receives and, at process exit, writes "<pushes> <pops> <names>" to the file named
 * by SBX_NVTX_COUNT_OUT. Built by tests/test_trace.py with gcc; loaded by NVTX through
 * NVTX_INJECTION64_PATH. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <nvtx3/nvToolsExt.h>

static int g_push, g_pop;
static char g_names[4096];

static int count_push(const char* msg) {
    g_push++;
    if (msg && strlen(g_names) + strlen(msg) + 2 < sizeof(g_names)) {
        strcat(g_names, msg);
        strcat(g_names, ",");
    }
    return 0;
}
static int count_pop(void) {
    g_pop++;
    return 0;
}
static void report(void) {
    const char* path = getenv("SBX_NVTX_COUNT_OUT");
    FILE* f = path ? fopen(path, "w") : NULL;
    if (!f) return;
    fprintf(f, "%d %d %s\n", g_push, g_pop, g_names);
    fclose(f);
}

int InitializeInjectionNvtx2(NvtxGetExportTableFunc_t getExportTable) {
    const NvtxExportTableCallbacks* cb = (const NvtxExportTableCallbacks*)getExportTable(NVTX_ETID_CALLBACKS);
    NvtxFunctionTable table = 0;
    unsigned int size = 0;
    if (!cb || !cb->GetModuleFunctionTable(NVTX_CB_MODULE_CORE, &table, &size)) return 0;
    if (size <= NVTX_CBID_CORE_RangePop) return 0;
    *table[NVTX_CBID_CORE_RangePushA] = (NvtxFunctionPointer)count_push;
    *table[NVTX_CBID_CORE_RangePop] = (NvtxFunctionPointer)count_pop;
    atexit(report);
    return 1;
}
