"""nvcc compiles a host function template that calls a __device__-only
function template without a diagnostic, and the call then does nothing on
the host (a workspace layout computed that way handed kernels garbage
pointers).  This scan of the CUDA sources fails when host code -- a function
not marked __global__ / __device__ / IPCB_D / IPCB_HD -- calls a helper that
is device-only (CPU)."""
import glob
import os
import re

CSRC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "ipc_warp_b200", "csrc")

_DEF = re.compile(r"^(template\s*<[^>]*>\s*)?(static\s+|inline\s+|constexpr\s+)*[\w:<>,\s\*&]+?\b(\w+)\s*\(")


def device_only(sources):
    """Names defined device-only and never as a host lambda (a member
    function and a host lambda may share a name)."""
    names, host = set(), set()
    for text in sources.values():
        for line in text.split("\n"):
            if "__host__" in line or "IPCB_HD" in line:
                continue
            m = re.search(r"(IPCB_D|__device__)(?:\s+__forceinline__)?\s+(?:inline\s+)?"
                          r"[\w:<>,\s\*&]+?\b(\w+)\s*\(", line)
            if m:
                names.add(m.group(2))
        host.update(re.findall(r"\bauto\s+(\w+)\s*=\s*\[", text))
    return names - host


def host_calls(text, dev):
    """(line, helper, host function) for calls of device-only helpers in host functions."""
    out = []
    lines = text.split("\n")
    depth, host, name, entered = 0, False, "", False
    for ln, line in enumerate(lines, 1):
        stripped = line.strip()
        if depth == 0 and not stripped.startswith(("//", "#")):
            head = line if "(" in line else ""
            prev = lines[ln - 2] if ln >= 2 else ""
            marked = any(k in head or k in prev for k in ("__global__", "IPCB_D", "IPCB_HD", "__device__"))
            if not host and head and _DEF.match(head) and not marked and "=" not in head.split("(")[0]:
                host, name, entered = True, head.strip()[:60], False
        if host:
            for d in dev:
                if re.search(r"\b" + d + r"\s*(<[^;()]*>)?\s*\(", line) and "<<<" not in line:
                    if not re.search(r"\b" + d + r"\s*(<[^;()]*>)?\s*\(", name):
                        out.append((ln, d, name))
        # namespace and extern "C" braces do not nest functions
        if not re.match(r'^\s*(namespace\b.*\{|extern\s+"C"\s*\{|\}\s*//\s*(namespace|extern))', line):
            depth += line.count("{") - line.count("}")
            if "{" in line:
                entered = True
        if depth == 0 and (entered or line.rstrip().endswith(";")):
            host = False  # the function body ended, or it was a declaration
    return out


def test_host_code_calls_no_device_only_helper():
    sources = {f: open(f).read() for f in glob.glob(os.path.join(CSRC, "*.cu*"))}
    dev = device_only(sources)
    assert len(dev) > 50
    bad = [(os.path.basename(f), *hit) for f, t in sources.items() if f.endswith(".cu") for hit in host_calls(t, dev)]
    assert not bad, bad


def test_scan_catches_a_host_call_of_a_device_template():
    text = ("namespace ipcb {\nnamespace {\ntemplate <class S>\nIPCB_D int helper(int a) { return a + 1; }\n\n"
            "template <class S>\nint launch(int n) {\n  int k = helper<S>(n);\n  return k;\n}\n"
            "}  // namespace\n}  // namespace ipcb\n")
    hits = host_calls(text, device_only({"x.cu": text}))
    assert [(h[1]) for h in hits] == ["helper"]
