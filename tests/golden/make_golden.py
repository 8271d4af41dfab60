"""Extract hom3's golden grid vectors into tests/golden/hierarchical_neighbors.json.

Reads hom3's own test file as text (it cannot be compiled here: Eigen, Boost
and gtest are absent) and copies out the expected values it asserts:

* hierarchical_container_test.cpp:43-49   -- grid size 73 for a level-2 3D cube
* hierarchical_container_test.cpp:58-82   -- children of nodes 0 and 1
* hierarchical_container_test.cpp:102-109 -- leaf flags (nodes >= 9 are leaves)
* hierarchical_container_test.cpp:134-147 -- same-level neighbours, 3D level 2
* hierarchical_container_test.cpp:212-274 -- same-level neighbours, 2D level 3

It also writes tests/golden/reference_files.json: the line count of every
source file of hom3 (.hpp, .cpp, .h, CMakeLists.txt), against which
tests/test_citations.py checks that each file:line citation in this
repository names lines that exist.

Run once in a checkout that has the hom3 sources (the path is required):
    python tests/golden/make_golden.py /path/to/hom3
"""
import json
import os
import re
import sys

INV = "eIdx"


def parse(src: str):
    out = {}
    m = re.search(r"EXPECT_EQ\(grid\.size\(\), Ind\{(\d+)\}\)", src)
    out["size_3d_level2"] = int(m.group(1))
    childs = re.findall(r"std::array<SInd, 8> childs_\d = \{\{([^}]*)\}\}", src)
    out["children_of_0"] = [int(x) for x in childs[0].split(",")]
    out["children_of_1"] = [int(x) for x in childs[1].split(",")]
    m = re.search(r"return nIdx < NodeIdx\{(\d+)\} \? false : true;", src)
    out["first_leaf_3d_level2"] = int(m.group(1))

    def vals(s):
        return [None if t.strip() == INV else int(t) for t in s.split(",")]

    # 3D table: lines like {{ eIdx,    2, eIdx,    3, eIdx,    5 }},  // nghbrs1
    block3 = src[src.index("auto nodeNghbrs = std::vector<std::array<Ind, 6>>"):]
    block3 = block3[: block3.index("});")]
    rows3 = re.findall(r"\{\{([^}]*)\}\},?\s*//\s*nghbrs(\d+)", block3)
    out["neighbors_3d_level2"] = {int(n): vals(r) for r, n in rows3}
    # 2D table: lines like {  1, {{ eIdx,    2, eIdx,    3 }}},
    block2 = src[src.index("auto nodeNghbrs = std::vector<nghbrIds<2>>"):]
    block2 = block2[: block2.index("});")]
    rows2 = re.findall(r"\{\s*(\d+),\s*\{\{([^}]*)\}\}\}", block2)
    out["neighbors_2d_level3"] = [[int(n), vals(r)] for n, r in rows2]
    return out


def file_lengths(root: str):
    """{path relative to the hom3 checkout: number of lines} of its sources."""
    out = {}
    for dp, dn, fn in os.walk(root):
        dn[:] = sorted(d for d in dn if not d.startswith("."))
        for f in sorted(fn):
            if f.endswith((".hpp", ".cpp", ".h")) or f == "CMakeLists.txt":
                full = os.path.join(dp, f)
                with open(full, errors="replace") as fh:
                    out[os.path.relpath(full, root)] = sum(1 for _ in fh)
    return out


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py /path/to/hom3")
    root = sys.argv[1]
    path = os.path.join(root, "src/containers/hierarchical/tests/hierarchical_container_test.cpp")
    with open(path) as f:
        data = parse(f.read())
    data["source"] = "src/containers/hierarchical/tests/hierarchical_container_test.cpp (hom3)"
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "hierarchical_neighbors.json")
    with open(dst, "w") as f:
        json.dump(data, f, indent=1)
    print("wrote", dst, {k: (len(v) if hasattr(v, "__len__") else v) for k, v in data.items()})
    lens = file_lengths(root)
    dst2 = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_files.json")
    with open(dst2, "w") as f:
        json.dump({"source": "line counts of hom3's source files", "files": lens}, f, indent=0, sort_keys=True)
    print("wrote", dst2, len(lens), "files")


if __name__ == "__main__":
    main()
