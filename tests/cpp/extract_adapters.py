"""Writes the adapter classes of INTEGRATION.md (its C++ blocks that define
classes) into one header, so the integration test compiles exactly the code
the document shows.  TEST INFRASTRUCTURE."""
import re
import sys

src = open(sys.argv[1]).read()
blocks = re.findall(r"```cpp\n(.*?)```", src, flags=re.S)
keep = [b for b in blocks if re.search(r"\bclass \w+B200\b", b)]
if not keep:
    sys.exit("no adapter classes found")
with open(sys.argv[2], "w") as f:
    f.write("// generated from INTEGRATION.md by tests/cpp/extract_adapters.py\n#pragma once\n")
    for b in keep:
        f.write(b + "\n")
