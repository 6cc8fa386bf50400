"""Write g++-compatible copies of two reference engine files into oracle/_ref/.

The reference engine targets Clang 18.  Two spots do not compile with g++ 13:

* engine/infra/Scheduler.cpp:86-91 wraps std::atomic members in an anonymous
  struct (a Clang extension).  The copy drops the wrapper so the members become
  plain members of Scheduler::Impl (only their cache-line padding changes).
* engine/storage/RestrictionLogic.cpp:20-36 builds bit masks with Clang's
  `ext_vector_type(bool)`.  The copy computes the same mask with a scalar loop
  over the GCC vector lanes.

Nothing is written outside oracle/_ref/, and the reference sources are only read.
This is test infrastructure for the oracle, not part of the product.
"""
import pathlib
import re
import sys

if len(sys.argv) != 3:
    sys.exit("usage: patch_ref.py <reference source root> <output dir>  (oracle/Makefile passes both)")
REF = pathlib.Path(sys.argv[1])
OUT = pathlib.Path(sys.argv[2])


def patch_scheduler(text: str) -> str:
    lines = text.splitlines(keepends=True)
    out, skip_close = [], False
    for line in lines:
        if "struct alignas(hardwareCachelineSize) {" in line:
            skip_close = True
            continue
        if skip_close and line.strip() == "};":
            skip_close = False
            continue
        out.append(line)
    assert not skip_close, "Scheduler.cpp: anonymous struct end not found"
    return "".join(out)


def patch_restriction(text: str) -> str:
    text, n1 = re.subn(r"typedef bool mask_vector __attribute__\(\(ext_vector_type\(vector_elements\)\)\);\n", "", text)
    body = re.compile(
        r"(static inline uint64_t movemask\(const T& vec\) \{\n)(.*?)(\n\})", re.S)
    text, n2 = body.subn(
        lambda m: m.group(1)
        + "    uint64_t result = 0;\n"
        + "    for (size_t i = 0; i < vector_elements; i++)\n"
        + "        result |= uint64_t(vec[i] != 0) << i;\n"
        + "    return result;"
        + m.group(3), text, count=1)
    assert n1 == 1 and n2 == 1, (n1, n2)
    return text


def main() -> None:
    OUT.mkdir(parents=True, exist_ok=True)
    sched = (REF / "engine/infra/Scheduler.cpp").read_text()
    (OUT / "Scheduler.cpp").write_text(patch_scheduler(sched))
    rl = (REF / "engine/storage/RestrictionLogic.cpp").read_text()
    (OUT / "RestrictionLogic.cpp").write_text(patch_restriction(rl))


if __name__ == "__main__":
    main()
