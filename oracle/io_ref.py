"""ORACLE — test infrastructure only.  A restatement in Python of the reference's
frame and lineage writers, against which tests/ compare the library's files:

  writeCells (ABM-3d/ABM-3d-cpp/include/utils.hpp:153-198; ABM-2d the same with the
  group in column 16): every parameter of the std::map (so in sorted key order) as
  "# key = value", then per cell the ID and group columns cast to int, the columns
  between them streamed as doubles under setprecision(10) (the default float field,
  i.e. printf "%.10g"), the write_other_cols columns as int (type 0) or double, each
  value followed by a tab, the last tab of a row replaced by the newline.

  writeLineage (utils.hpp:296-311): "i<TAB>parent" per cell ID.

The product library never imports anything under oracle/.
"""

GROUP_COL = {3: 20, 2: 16}


def write_cells_text(cells, params, extra_cols=None, dims=3):
    out = []
    for key in sorted(params):
        out.append("# %s = %s\n" % (key, params[key]))
    group = GROUP_COL[dims]
    extra = extra_cols or {}
    n, ncols = len(cells), len(cells[0]) if len(cells) else 0
    for i in range(n):
        row = ""
        for j in range(ncols):
            v = float(cells[i][j])
            if j == 0 or j == group:
                row += "%d\t" % int(v)
            elif 0 < j < group:
                row += "%.10g\t" % v
            elif j in extra:
                row += ("%d\t" % int(v)) if extra[j] == 0 else ("%.10g\t" % v)
        out.append(row[:-1] + "\n")
    return "".join(out)


def lineage_text(parents):
    return "".join("%d\t%d\n" % (i, p) for i, p in enumerate(parents))
