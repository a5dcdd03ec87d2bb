# Install (1), uninstall (0) or update (2) the B200 package in a LAMMPS
# src/ tree:  cd src/B200 && sh Install.sh 1   (with this directory copied
# or linked there as src/B200)
#
# B200_ROOT must point at the lammps_b200 checkout whose libb200md.so is
# built (python lammps_b200/build.py); the package adds its include and
# library paths to src/Makefile.package.

mode=$1
files="b200_link.h b200_link.cpp pair_lj_cut_b200.h pair_lj_cut_b200.cpp
       pair_eam_b200.h pair_eam_b200.cpp fix_nve_b200.h fix_nve_b200.cpp
       verlet_b200.h verlet_b200.cpp dump_custom_b200.h dump_custom_b200.cpp"

if (test $mode = 1 || test $mode = 2) then
  if (test ! -e ../pair_eam.h) then
    echo "B200 needs the MANYBODY package: make yes-manybody first"
    exit 1
  fi
  for f in $files; do
    if (! cmp -s $f ../$f) then
      cp $f ..
      if (test $mode = 2) then echo "  updating src/$f"; fi
    fi
  done
  if (test -e ../Makefile.package) then
    sed -i -e 's|-I$(B200_ROOT)/include ||' -e 's|-L$(B200_ROOT)/lammps_b200/_lib ||' \
           -e 's|-lb200md ||' ../Makefile.package
    sed -i -e 's|^PKG_INC =[ \t]*|&-I$(B200_ROOT)/include |' \
           -e 's|^PKG_PATH =[ \t]*|&-L$(B200_ROOT)/lammps_b200/_lib |' \
           -e 's|^PKG_LIB =[ \t]*|&-lb200md |' ../Makefile.package
  fi
elif (test $mode = 0) then
  for f in $files; do rm -f ../$f; done
  if (test -e ../Makefile.package) then
    sed -i -e 's|-I$(B200_ROOT)/include ||' -e 's|-L$(B200_ROOT)/lammps_b200/_lib ||' \
           -e 's|-lb200md ||' ../Makefile.package
  fi
fi
