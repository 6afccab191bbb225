"""Build step: embeds the device headers of the aggregate kernel as C++ raw
string literals (jit_sources.inc), so the runtime can compile per-spec
kernels from them with NVRTC without the source tree being present."""
import os
import sys


def main(out, *paths):
    lines = ["// generated by embed_sources.py -- do not edit", "namespace vr { namespace jitsrc {"]
    names, vars_ = [], []
    for i, p in enumerate(paths):
        text = open(p).read()
        assert ')VRSRC"' not in text
        var = f"kSrc{i}"
        lines.append(f'static const char* const {var} = R"VRSRC({text})VRSRC";')
        names.append(os.path.basename(p))
        vars_.append(var)
    lines.append(f"static const int kNum = {len(paths)};")
    lines.append("static const char* const kNames[] = {" + ", ".join(f'"{n}"' for n in names) + "};")
    lines.append("static const char* const kTexts[] = {" + ", ".join(vars_) + "};")
    lines.append("}}  // namespace vr::jitsrc")
    tmp = out + ".tmp"
    with open(tmp, "w") as f:
        f.write("\n".join(lines) + "\n")
    os.replace(tmp, out)


if __name__ == "__main__":
    main(sys.argv[1], *sys.argv[2:])
