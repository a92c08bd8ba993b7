# Keep one side of every git conflict block: -v side=head | theirs.
/^<<<<<<< / { st = 1; next }
/^=======/  { if (st == 1) { st = 2; next } }
/^>>>>>>> / { if (st == 2) { st = 0; next } }
{ if (st == 0 || (st == 1 && side == "head") || (st == 2 && side == "theirs")) print }
