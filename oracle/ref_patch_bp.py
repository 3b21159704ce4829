"""Writes a copy of the reference's numa-BP.C that can be compared with the
oracle (test infrastructure; the copy goes to oracle/_ref/src, outside
version control).  The stock program leaves its inputs unset -- priors from
malloc (numa-BP.C:557), products and edge potentials zero-filled -- and its
-result block is empty (588-590).  The copy changes only those points:
  priors      vertex v: p0 = (float)(0.2 + 0.6 * ((37 v + 11) mod 101) / 101),
              p1 = 1 - p0 (in float), after the malloc;
  products    the current products start at 1 (after mapDataArray);
  potentials  every edge [[0.9, 0.1], [0.1, 0.9]] (after numa_alloc_local);
  -result     prints "prod v p0 p1" (%.9e) from the buffer holding the last
              round's products (the workers swap curr/next every round).
The edge pass and the frontier rules are the reference's, untouched.

  python ref_patch_bp.py <numa-BP.C> <out.C>"""
import sys

EDITS = [
    ("    VertexInfo *vertI = (VertexInfo *)malloc(sizeof(VertexInfo) * GA.n);\n",
     "    for (intT pmv = 0; pmv < GA.n; pmv++) {\n"
     "        vertI[pmv].potential[0] = (float)(0.2 + 0.6 * (double)((37 * (long)pmv + 11) % 101) / 101.0);\n"
     "        vertI[pmv].potential[1] = 1.0f - vertI[pmv].potential[0];\n"
     "    }\n"),
    ("    VertexData *vertD_next = (VertexData *)mapDataArray(numOfNode, sizeArr, sizeof(VertexData));\n",
     "    for (intT pmv = 0; pmv < GA.n; pmv++) { vertD_curr[pmv].product[0] = 1.0f; vertD_curr[pmv].product[1] = 1.0f; }\n"),
    ("    EdgeWeight *edgeW = (EdgeWeight *)numa_alloc_local(sizeof(EdgeWeight) * numLocalEdge);\n",
     "    for (intT pme = 0; pme < numLocalEdge; pme++) {\n"
     "        edgeW[pme].potential[0][0] = 0.9f; edgeW[pme].potential[0][1] = 0.1f;\n"
     "        edgeW[pme].potential[1][0] = 0.1f; edgeW[pme].potential[1][1] = 0.9f;\n"
     "    }\n"),
    ("    if (needResult) {\n",
     "        VertexData *pm_last = (maxIter % 2) ? vertD_next : vertD_curr;\n"
     "        for (intT pmv = 0; pmv < GA.n; pmv++)\n"
     "            printf(\"prod %ld %.9e %.9e\\n\", (long)pmv, (double)pm_last[pmv].product[0],\n"
     "                   (double)pm_last[pmv].product[1]);\n"),
]


def main(src, dst):
    text = open(src).read()
    for anchor, insert in EDITS:
        if text.count(anchor) != 1:
            raise SystemExit("anchor not found exactly once: %r" % anchor)
        text = text.replace(anchor, anchor + insert)
    with open(dst, "w") as f:
        f.write(text)


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2])
