# extract_fns.awk -- copies the named functions of a reference header
# (fns="a,b,c"), with the header's preamble (everything before the line that
# opens namespace `ns`, minus the thrust / cub includes that only its host
# launch code needs), into a header that a host build can include.  Used by
# the Makefile on the reference sources; its output goes to oracle/_ref/inc.
BEGIN {
    n = split(fns, want, ",")
    for (i = 1; i <= n; ++i) wanted[want[i]] = 1
    pre = 1; depth = 0; cap = 0; opened = 0
}
{ sub(/\r$/, "") }
pre && $0 ~ ("^[ \t]*namespace[ \t]+" ns "[ \t]*\\{") { pre = 0; print "namespace " ns " {"; next }
pre { if ($0 !~ /#include[ \t]*<(thrust|cub)\//) print; next }
!cap {
    for (f in wanted)
        if ($0 ~ ("(__global__|__device__|__host__).*[ \t*&]" f "[ \t]*\\(")) { cap = 1; depth = 0; opened = 0 }
}
cap {
    print
    line = $0
    sub(/\/\/.*/, "", line)
    o = gsub(/\{/, "{", line); c = gsub(/\}/, "}", line)
    depth += o - c
    if (o > 0) opened = 1
    if (opened && depth <= 0) { cap = 0; print "" }
}
END { print "}  // namespace " ns }
