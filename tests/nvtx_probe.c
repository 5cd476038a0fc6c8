/* nvtx_probe.c -- a minimal NVTX injection library for the tracing test.
 *
 * NVTX3 (header-only, compiled into libcatabra_b200.so) loads the library
 * named by NVTX_INJECTION64_PATH on its first call and hands it the callback
 * tables; this one fills the domain create / range push / range pop slots
 * and records every call as a text line ("domain <name>", "push <message>",
 * "pop"), which nvtx_probe_dump returns.  Test infrastructure only. */
#include <stdio.h>
#include <string.h>

#include <nvtx3/nvToolsExt.h>

static char g_log[1 << 16];
static size_t g_len;
static int g_depth;

static void note(const char* kind, const char* text) {
    char line[400];
    int k = snprintf(line, sizeof line, "%s%s%s\n", kind, text ? " " : "", text ? text : "");
    if (k > 0 && g_len + (size_t)k + 1 < sizeof g_log) {
        memcpy(g_log + g_len, line, (size_t)k);
        g_len += (size_t)k;
        g_log[g_len] = 0;
    }
}
static nvtxDomainHandle_t NVTX_API probe_domain_create(const char* name) {
    note("domain", name);
    return (nvtxDomainHandle_t)(void*)&g_depth;
}
static int NVTX_API probe_push(nvtxDomainHandle_t d, const nvtxEventAttributes_t* a) {
    (void)d;
    note("push", (a && a->messageType == NVTX_MESSAGE_TYPE_ASCII) ? a->message.ascii : "?");
    return ++g_depth;
}
static int NVTX_API probe_pop(nvtxDomainHandle_t d) {
    (void)d;
    note("pop", NULL);
    return g_depth--;
}

int nvtx_probe_dump(char* buf, int len) {
    snprintf(buf, (size_t)len, "%s", g_log);
    return (int)g_len;
}

int InitializeInjectionNvtx2(NvtxGetExportTableFunc_t get) {
    const NvtxExportTableCallbacks* cb = (const NvtxExportTableCallbacks*)get(NVTX_ETID_CALLBACKS);
    NvtxFunctionTable t = 0;
    unsigned int size = 0;
    if (!cb || !cb->GetModuleFunctionTable(NVTX_CB_MODULE_CORE2, &t, &size) || !t) return 0;
    if (size > NVTX_CBID_CORE2_DomainCreateA) *t[NVTX_CBID_CORE2_DomainCreateA] = (NvtxFunctionPointer)probe_domain_create;
    if (size > NVTX_CBID_CORE2_DomainRangePushEx) *t[NVTX_CBID_CORE2_DomainRangePushEx] = (NvtxFunctionPointer)probe_push;
    if (size > NVTX_CBID_CORE2_DomainRangePop) *t[NVTX_CBID_CORE2_DomainRangePop] = (NvtxFunctionPointer)probe_pop;
    return 1;
}
